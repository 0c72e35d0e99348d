// Per-target dual-tree traversal: the exact far / near lists of the
// symmetric walk (_interactions_impl.py:1119-1905, 2600-3558; result
// layouts :3561-3837) produced row by row, without a pair log, an atomic
// scatter or a per-row sort.
//
// The reference's walk refines canonical node pairs breadth first from
// (root, root).  Seen from one node t, the visited pairs {t, s} are:
//  * the pairs inherited from the parent p: every {p, s} that the walk
//    refined by splitting p (the split rule on the canonical orientation,
//    :1444-1454), plus the sibling pair {L, R} that the self pair {p, p}
//    produces;
//  * and, recursively, the children {t, s.left}, {t, s.right} of every
//    visited {t, s} refined by splitting s.
// So t's pairs follow from its parent's "split on my side" list S_p alone,
// and the nodes can be processed top down, one warp per target, each warp
// evaluating the MAC (:338-395) in the reference's fp32 order on exactly the
// pairs the reference evaluates (every unordered pair twice, once from each
// side).
//
// Row order without sorting: the candidates of one target are disjoint
// subtrees, and a warp walks them in Morton order (an ordered depth-first
// expansion: it pops the 32 leftmost pending candidates, emits the leading
// ones that are resolved, and pushes the rest back in order).  For disjoint
// Karras ranges, Morton order is id order within internal nodes (an internal
// node's id is the first or last leaf of its range) and within leaves (id =
// num_internal + leaf index), and every internal id is below every leaf id.
// So a far row in ascending id order is its internal entries in Morton order
// followed by its leaf entries in Morton order, and a near row (leaves only)
// is the Morton order itself.  The warp stages the two far classes and the
// near entries separately; every flushed chunk is keyed by (row, class,
// first id), and one sort of the chunk records (not of the entries) puts all
// rows in their final, ascending order.
//
// Work balance: a target whose expansion runs longer than a step budget, or
// whose ordered stack fills, spills its pending candidates (in order) and
// hands them to other warps as continuation pieces.  Pieces of one target
// cover disjoint Morton intervals, so their chunks still sort into place.
// A node's own "split on my side" list is compacted into one Morton-ordered
// array when its last piece ends, and only then may its children start.
// One persistent launch processes every level: warps take pieces first,
// then targets in level order, and wait (bounded) only on a parent that is
// still in progress.
#include "rows.cuh"
#include "scan.cuh"
#include "sort.cuh"

namespace ygx {
namespace {

struct __align__(16) TwRec {
  float4 c;  // center x, y, z; MAC extent
  int4 k;    // left, right (-1 for leaves), leaf position (-1 internal), first leaf index
};

enum TwMac { kTwBH = 0, kTwDehnen = 1, kTwEngblom = 2 };

// Candidate entry (64 bits): node id (31 bits) | generation << 32 (12 bits)
// | state << 44 (2 bits) | before << 46.  States: 0 pending, 1 far, 2 near,
// 3 split on the target's side.  "before": the node's range starts before
// the target's (counted for the children's sibling insertion point).
__device__ __forceinline__ unsigned long long tw_ent(int s, int gen, int state, int before) {
  return (unsigned long long)(uint32_t)s | ((unsigned long long)(uint32_t)gen << 32) |
         ((unsigned long long)(uint32_t)state << 44) | ((unsigned long long)(uint32_t)before << 46);
}
__device__ __forceinline__ int tw_s(unsigned long long e) { return (int)(e & 0x7fffffffull); }
__device__ __forceinline__ int tw_gen(unsigned long long e) { return (int)((e >> 32) & 0xfffull); }
__device__ __forceinline__ int tw_state(unsigned long long e) { return (int)((e >> 44) & 3ull); }
__device__ __forceinline__ int tw_before(unsigned long long e) { return (int)((e >> 46) & 1ull); }
constexpr unsigned long long kTwPendingMask = 0xfffffffffffull;  // id + generation

constexpr int kTwWarps = 8;
constexpr int kTwThreads = kTwWarps * 32;
constexpr int kTwBlocksPerSM = 4;
constexpr int kTwStk = 256;    // ordered stack entries per warp
constexpr int kTwStgF = 128;   // staging of far-internal / far-leaf / near entries
constexpr int kTwStgS = 256;   // staging of split-list entries
constexpr int kTwHist = 256;   // generations counted per CTA (pair generations < 2 x depth)
constexpr int kTwCmpMax = 256; // chunks a split list may have before compaction
constexpr int kTwSpillGroup = 8;
constexpr int kTwInhGroup = 64;

// A warp's current allocation block in one pool (kept in shared memory):
// pool space is claimed from the global cursor in blocks, so most flushes
// need no global atomic.
struct TwBlk {
  unsigned long long cur, end;
};
struct TwBlkSet {
  TwBlk far, near_, s, far_r, near_r, s_r;
};
// A warp's counters (lane 0 only): decisions per side, cycles on pieces and
// waiting, pieces, 32-wide steps and the candidates they held.
struct TwWarpStats {
  unsigned long long acc, near_, ref, busy, idle, pieces, steps, lanes;
};
constexpr unsigned kTwNoTicket = 0xffffffffu;
struct TwWarpSmem {
  TwBlkSet al;  // the warp's allocation blocks
  TwWarpStats st;
  long long t_mark;  // clock at the last piece boundary
  unsigned long long stk[kTwStk];
  unsigned long long stg_s[kTwStgS];
  int32_t stg_fi[kTwStgF];
  int32_t stg_fl[kTwStgF];
  int32_t stg_n[kTwStgF];
};
struct TwSmem {
  TwWarpSmem w[kTwWarps];
  unsigned int hist[kTwHist];
};

// Control block (zeroed before the walk).  Every counter that many warps
// update or poll sits on its own 128-byte line, so the atomics of one do not
// queue behind traffic on another.
#define TW_LINE(type, name) \
  type name;                \
  char name##_pad[128 - sizeof(type)]
struct __align__(128) TwCtl {
  TW_LINE(unsigned long long, far_cur);  // pool cursors (entries)
  TW_LINE(unsigned long long, near_cur);
  TW_LINE(unsigned long long, s_cur);
  TW_LINE(unsigned long long, spill_cur);
  TW_LINE(unsigned int, far_rec_cur);    // chunk record cursors
  TW_LINE(unsigned int, near_rec_cur);
  TW_LINE(unsigned int, s_rec_cur);
  TW_LINE(unsigned int, q_head);         // continuation queue: tickets taken
  TW_LINE(unsigned int, q_tail);         // slots filled
  TW_LINE(unsigned int, tick);           // next target
  TW_LINE(int, work);                    // targets + pieces outstanding
  // written once per warp at exit
  unsigned long long acc_sides, near_sides, ref_sides;  // decision counts (per side)
  unsigned long long busy_cycles, idle_cycles, pieces;  // where the warps' time went
  unsigned long long steps, lanes;  // 32-wide steps run, candidates they held
  unsigned int max_cmp;                                 // most chunks of one split list
  unsigned int pad[3];
};
#undef TW_LINE

struct TwPiece {
  long long spill_off;
  int t;
  int spill_cnt;
  int inh_b, inh_e;
};

struct TwChunk {  // a flushed far / near chunk
  long long off;
  int cnt;
  int t;
};
struct TwSChunk {  // a flushed split-list chunk (linked per node)
  long long off;
  int cnt;
  unsigned int key;  // first leaf of the chunk's first entry
  int next;
  int pad;
};

struct TwArgs {
  const TwRec* recs;
  const int32_t* nbl;        // nodes in level order
  const int32_t* parent;
  const int32_t* level;      // node depth
  const int32_t* rank;       // position in nbl
  int32_t ni, total, lo, n_targets;
  float theta_sq, theta;
  // per node
  long long* s_off;
  int32_t* s_cnt;
  int32_t* s_ins;
  int32_t* s_head;
  int32_t* s_nch;
  int32_t* pieces_left;
  int32_t* done;
  int32_t* far_cnt;   // per node
  int32_t* near_cnt;  // per leaf position
  // pools
  int32_t* far_pool;
  int32_t* near_pool;
  unsigned long long* s_pool;
  unsigned long long* spill;
  unsigned long long far_cap, near_cap, s_cap, spill_cap;
  unsigned long long* far_keys;
  TwChunk* far_recs;
  unsigned long long* near_keys;
  TwChunk* near_recs;
  TwSChunk* s_recs;
  unsigned int far_rec_cap, near_rec_cap, s_rec_cap, q_cap;
  TwPiece* queue;
  unsigned int* q_ready;
  unsigned int* gen_hist;  // global, kTwHist words
  TwCtl* ctl;
  uint32_t* status;
  uint32_t spin_limit;
  int budget;
  unsigned long long blk_entries;  // pool block (entries) per claim
  unsigned int blk_records;        // record block per claim
  // unordered walks with predicted row capacities: a chunk that fits its
  // row's capacity is written in place at pad[row] + its offset in the row
  const int32_t* far_rcap;   // per node (nullptr: no prediction)
  const int32_t* near_rcap;  // per leaf position
  const int64_t* pad_far;    // padded row starts, per node / leaf position
  const int64_t* pad_near;
  int32_t* far_raw;
  int32_t* near_raw;
  unsigned* first_ovf_far;   // smallest in-row offset that went to the pool
  unsigned* first_ovf_near;
};

// Takes n slots from the warp's block *b (in shared memory, touched by lane
// 0 only), claiming a new block of at least `blk` slots from the global
// cursor when *b is short.  Warp-collective; false (and the block dropped)
// when the pool is out of room.
template <typename U>
__device__ __forceinline__ bool tw_take(TwBlk* b, unsigned long long n, unsigned long long blk,
                                        U* cursor, unsigned long long cap, int lane,
                                        unsigned long long* off) {
  unsigned long long o = 0;
  int ok = 1;
  if (lane == 0) {
    if (b->cur + n > b->end) {
      const unsigned long long sz = n > blk ? n : blk;
      const unsigned long long g = (unsigned long long)atomicAdd(cursor, (U)sz);
      if (g + sz > cap) {
        b->cur = b->end = 0;
        ok = 0;
      } else {
        b->cur = g;
        b->end = g + sz;
      }
    }
    if (ok) {
      o = b->cur;
      b->cur += n;
    }
  }
  *off = __shfl_sync(0xffffffffu, o, 0);
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__device__ __forceinline__ unsigned lanemask_lt_() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ int ld_acquire_i32(const int32_t* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_volatile_u32_(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_volatile_i32_(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_i32(int32_t* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------------------
// setup

// first[v]: index of the first (leftmost) leaf under node v.  Each leaf
// climbs while it is its parent's left child.
__global__ void k_tw_first_leaf(const int32_t* __restrict__ parent, const int32_t* __restrict__ left,
                                int32_t ni, int32_t total, int32_t* __restrict__ first) {
  for (int32_t v = ni + blockIdx.x * blockDim.x + threadIdx.x; v < total;
       v += gridDim.x * blockDim.x) {
    const int32_t j = v - ni;
    first[v] = j;
    int32_t c = v;
    for (int guard = 0; guard < 128; ++guard) {
      const int32_t p = parent[c];
      if (p < 0 || p >= ni || left[p] != c) break;
      first[p] = j;
      c = p;
    }
  }
}

__global__ void k_tw_recs(const float* __restrict__ center, const float* __restrict__ radius,
                          const float* __restrict__ max_extent, const int32_t* __restrict__ left32,
                          const int32_t* __restrict__ right32, const int32_t* __restrict__ leafpos,
                          const int32_t* __restrict__ first, int32_t total, int mac,
                          float dehnen_scale, const int32_t* __restrict__ nbl,
                          int32_t* __restrict__ rank, TwRec* __restrict__ recs,
                          uint32_t* __restrict__ status) {
  for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    // _build_mac_extents (_interactions_impl.py:993-1061)
    float e = mac == kTwBH ? max_extent[k] : radius[k];
    if (mac == kTwDehnen) e = __fmul_rn(dehnen_scale, e);
    if (!(e > 0.0f)) raise_flag(status, kFlagBadInput);
    TwRec r;
    r.c = make_float4(center[3 * k], center[3 * k + 1], center[3 * k + 2], e);
    r.k = make_int4(left32[k], right32[k], leafpos[k], first[k]);
    recs[k] = r;
    rank[nbl[k]] = k;
  }
}

// Root: done, empty split list.  Every other node: no chunks yet.
__global__ void k_tw_init_nodes(int32_t total, int32_t root, int32_t* __restrict__ s_head,
                                long long* __restrict__ s_off, int32_t* __restrict__ done) {
  for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    s_head[k] = -1;
    s_off[k] = 0;
    done[k] = k == root ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------
// the walk

// Warp-collective: writes the n staged int32 entries to `pool` and records
// the chunk, and counts the row.  The record's key: ordered walks, row |
// class | first id (the chunks are sorted by it); unordered walks, row |
// the chunk's offset within the row (taken by the count).  With a predicted
// row (raw != nullptr) the offset is taken first and a chunk that ends within
// the row's capacity rcap is written in place at raw[pad + offset] instead
// (no record); the others go to the pool, and first_ovf keeps the smallest
// offset that did.
template <bool kOrd>
__device__ __forceinline__ void tw_flush_rows(const int32_t* stg, int n, int lane, int t,
                                              unsigned long long key_hi, unsigned cls_bit,
                                              int32_t* pool, unsigned long long cap,
                                              unsigned long long* pool_cur, TwBlk* pb,
                                              unsigned long long* keys, TwChunk* recs,
                                              unsigned rec_cap, unsigned* rec_cur, TwBlk* rb,
                                              int32_t* cnt_row, int32_t* raw, int rcap,
                                              int64_t pad, unsigned* first_ovf,
                                              const TwArgs& a) {
  if (n == 0) return;
  unsigned long long off = 0, ri = 0;
  if (!kOrd && raw) {
    int within = 0;
    if (lane == 0) within = atomicAdd(cnt_row, n);
    within = __shfl_sync(0xffffffffu, within, 0);
    if ((long long)within + n <= (long long)rcap) {
      for (int k = lane; k < n; k += 32) raw[pad + within + k] = stg[k];
      return;
    }
    const bool fits = tw_take(pb, (unsigned long long)n, a.blk_entries, pool_cur, cap, lane, &off) &&
                      tw_take(rb, 1ull, a.blk_records, rec_cur, rec_cap, lane, &ri);
    if (fits) {
      for (int k = lane; k < n; k += 32) pool[off + k] = stg[k];
      if (lane == 0) {
        keys[ri] = key_hi | (unsigned long long)(uint32_t)within;
        TwChunk c;
        c.off = (long long)off;
        c.cnt = n;
        c.t = t;
        recs[ri] = c;
        atomicMin(first_ovf, (unsigned)within);
      }
    } else if (lane == 0) {
      raise_flag(a.status, kFlagLogOverflow);
    }
    return;
  }
  const bool ok = tw_take(pb, (unsigned long long)n, a.blk_entries, pool_cur, cap, lane, &off) &&
                  tw_take(rb, 1ull, a.blk_records, rec_cur, rec_cap, lane, &ri);
  if (ok) {
    for (int k = lane; k < n; k += 32) pool[off + k] = stg[k];
    if (lane == 0) {
      const int within = atomicAdd(cnt_row, n);
      keys[ri] = key_hi | (kOrd ? (cls_bit | (unsigned long long)(uint32_t)stg[0])
                                : (unsigned long long)(uint32_t)within);
      TwChunk c;
      c.off = (long long)off;
      c.cnt = n;
      c.t = t;
      recs[ri] = c;
    }
  } else if (lane == 0) {
    raise_flag(a.status, kFlagLogOverflow);
  }
}

__device__ __forceinline__ void tw_flush_split(const unsigned long long* stg, int n, int lane, int t,
                                               const TwArgs& a, TwBlkSet& al) {
  if (n == 0) return;
  unsigned long long off = 0, ri = 0;
  const bool fits =
      tw_take(&al.s, (unsigned long long)n, a.blk_entries, &a.ctl->s_cur, a.s_cap, lane, &off) &&
      tw_take(&al.s_r, 1ull, a.blk_records, &a.ctl->s_rec_cur, a.s_rec_cap, lane, &ri);
  int before = 0;
  for (int k = lane; k < n; k += 32) {
    const unsigned long long e = stg[k];
    before += tw_before(e);
    if (fits) a.s_pool[off + k] = e & kTwPendingMask;  // stored as pending entries
  }
  for (int o = 16; o > 0; o >>= 1) before += __shfl_xor_sync(0xffffffffu, before, o);
  if (lane == 0) {
    if (fits) {
      TwSChunk c;
      c.off = (long long)off;
      c.cnt = n;
      c.key = (unsigned)a.recs[tw_s(stg[0])].k.w;
      c.pad = 0;
      c.next = atomicExch(&a.s_head[t], (int)ri);
      a.s_recs[ri] = c;
      atomicAdd(&a.s_cnt[t], n);
      atomicAdd(&a.s_ins[t], before);
      atomicAdd(&a.s_nch[t], 1);
    } else {
      raise_flag(a.status, kFlagLogOverflow);
    }
  }
}

// Warp-collective: compacts node t's split-list chunks into one array --
// in Morton order by their first leaf when kSortChunks (ordered walks; at
// most kTwCmpMax chunks), else in list order.  Called by the warp that ends
// t's last piece.
template <bool kSortChunks>
__device__ void tw_compact_split(int t, int lane, const TwArgs& a, unsigned long long* scratch) {
  const int nch = ld_volatile_i32_(&a.s_nch[t]);
  if (nch == 0) {
    if (lane == 0) a.s_off[t] = 0;
    return;
  }
  const int head = ld_volatile_i32_(&a.s_head[t]);
  if (nch == 1) {
    if (lane == 0) a.s_off[t] = a.s_recs[head].off;
    return;
  }
  if (lane == 0) atomicMax(&a.ctl->max_cmp, (unsigned)nch);
  if (kSortChunks) {
    if (nch > kTwCmpMax) {  // cannot order it here: report (the host falls back)
      if (lane == 0) {
        raise_flag(a.status, kFlagMalformed);
        a.s_cnt[t] = 0;  // children see an empty list (the result is discarded)
        a.s_ins[t] = 0;
      }
      return;
    }
    // collect (key << 32 | record) pairs; lane 0 walks the list
    if (lane == 0) {
      int r = head, k = 0;
      while (r >= 0 && k < nch) {
        const TwSChunk c = a.s_recs[r];
        scratch[k++] = ((unsigned long long)c.key << 32) | (unsigned)r;
        r = c.next;
      }
    }
    __syncwarp();
    // odd-even transposition sort of nch <= 256 keys (small; rare)
    for (int pass = 0; pass < nch; ++pass) {
      for (int i = 2 * lane + (pass & 1); i + 1 < nch; i += 64) {
        const unsigned long long x = scratch[i], y = scratch[i + 1];
        if (x > y) {
          scratch[i] = y;
          scratch[i + 1] = x;
        }
      }
      __syncwarp();
    }
  }
  const int total = ld_volatile_i32_(&a.s_cnt[t]);
  unsigned long long off = 0;
  if (lane == 0) off = atomicAdd(&a.ctl->s_cur, (unsigned long long)total);
  off = __shfl_sync(0xffffffffu, off, 0);
  if (off + (unsigned long long)total > a.s_cap) {
    if (lane == 0) {
      raise_flag(a.status, kFlagLogOverflow);
      a.s_cnt[t] = 0;
      a.s_ins[t] = 0;
    }
    return;
  }
  unsigned long long pos = off;
  int r = head;
  for (int k = 0; k < nch; ++k) {
    if (!kSortChunks && r < 0) break;
    const int ri = kSortChunks ? (int)(unsigned)(scratch[k] & 0xffffffffu) : r;
    const TwSChunk c = a.s_recs[ri];
    for (int e = lane; e < c.cnt; e += 32) a.s_pool[pos + e] = a.s_pool[c.off + e];
    pos += (unsigned long long)c.cnt;
    r = c.next;
  }
  if (lane == 0) a.s_off[t] = (long long)off;
}

// Warp-collective: the rest of this piece -- P pending outputs (lane l holds
// nout of them from index k0), then the ordered stack (top first), then the
// source remainder from `cur` -- is handed to other warps as continuation
// pieces, in groups.  Pieces of one target cover disjoint Morton intervals,
// so their output chunks sort into place whatever warp runs them.
__device__ void tw_hand_off(const TwArgs& a, int lane, int t, const TwPiece& pc, int cur,
                            int nout, int k0, unsigned long long o0, unsigned long long o1, int P,
                            const unsigned long long* stk, int stk_n) {
  const int E = P + stk_n;
  unsigned long long off = 0;
  if (lane == 0 && E > 0) off = atomicAdd(&a.ctl->spill_cur, (unsigned long long)E);
  off = __shfl_sync(0xffffffffu, off, 0);
  if (off + (unsigned long long)E > a.spill_cap) {
    if (lane == 0) raise_flag(a.status, kFlagLogOverflow);
    return;
  }
  if (nout >= 1) a.spill[off + k0] = o0;
  if (nout == 2) a.spill[off + k0 + 1] = o1;
  for (int j = lane; j < stk_n; j += 32) a.spill[off + P + j] = stk[stk_n - 1 - j];
  const int np_sp = (E + kTwSpillGroup - 1) / kTwSpillGroup;
  const int rem_sp = cur < pc.spill_cnt ? pc.spill_cnt - cur : 0;
  const int np_rs = (rem_sp + kTwSpillGroup - 1) / kTwSpillGroup;
  const int inh_from = pc.inh_b + (cur > pc.spill_cnt ? cur - pc.spill_cnt : 0);
  const int rem_in = pc.inh_e - inh_from;
  const int np_in = rem_in > 0 ? (rem_in + kTwInhGroup - 1) / kTwInhGroup : 0;
  const int np = np_sp + np_rs + np_in;
  if (np == 0) return;
  unsigned slot = 0;
  int n_ok = 0;
  if (lane == 0) {
    slot = atomicAdd(&a.ctl->q_tail, (unsigned)np);
    n_ok = slot >= a.q_cap ? 0 : (int)min((unsigned)np, a.q_cap - slot);
    if (n_ok < np) raise_flag(a.status, kFlagLogOverflow);
    // counted before any of them can be taken (and finished) by another warp
    if (n_ok > 0) {
      atomicAdd(&a.pieces_left[t], n_ok);
      atomicAdd(&a.ctl->work, n_ok);
    }
    __threadfence();
  }
  slot = __shfl_sync(0xffffffffu, slot, 0);
  n_ok = __shfl_sync(0xffffffffu, n_ok, 0);
  __syncwarp();
  for (int k = lane; k < n_ok; k += 32) {
    TwPiece q;
    q.t = t;
    if (k < np_sp) {
      q.spill_off = (long long)(off + (unsigned long long)k * kTwSpillGroup);
      q.spill_cnt = min(kTwSpillGroup, E - k * kTwSpillGroup);
      q.inh_b = q.inh_e = 0;
    } else if (k < np_sp + np_rs) {
      const int j = k - np_sp;
      q.spill_off = pc.spill_off + cur + (long long)j * kTwSpillGroup;
      q.spill_cnt = min(kTwSpillGroup, rem_sp - j * kTwSpillGroup);
      q.inh_b = q.inh_e = 0;
    } else {
      const int j = k - np_sp - np_rs;
      q.spill_off = 0;
      q.spill_cnt = 0;
      q.inh_b = inh_from + j * kTwInhGroup;
      q.inh_e = min(pc.inh_e, q.inh_b + kTwInhGroup);
    }
    a.queue[slot + k] = q;
    __threadfence();
    atomicExch(&a.q_ready[slot + k], 1u);
  }
}

// kOrd: rows in ascending order straight from the walk (the ordered
// expansion above).  Otherwise every resolved candidate is emitted at once
// and only the children of refined ones go back on the stack (no re-popped
// lanes, no ordered push); the rows are sorted after the walk.
//
// Each step is software-pipelined: once this window's outputs are on the
// stack, the next window is popped and its node records are requested, and
// only then are this window's resolved entries staged (and flushed), so the
// record gathers of step k + 1 overlap the emission work of step k.
template <int kMac, bool kOrd>
__global__ void __launch_bounds__(kTwThreads, kTwBlocksPerSM) k_tw_walk(TwArgs a) {
  extern __shared__ __align__(16) unsigned char tw_smem_raw[];
  TwSmem& sm = *reinterpret_cast<TwSmem*>(tw_smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  TwWarpSmem& W = sm.w[warp];
  for (int i = threadIdx.x; i < kTwHist; i += kTwThreads) sm.hist[i] = 0;
  TwBlkSet& al = W.al;
  if (lane == 0) {
    al.far = al.near_ = al.s = al.far_r = al.near_r = al.s_r = TwBlk{0ull, 0ull};
    W.st = TwWarpStats{0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
    W.t_mark = clock64();
  }
  __syncthreads();
  const unsigned lt = lanemask_lt_();
  int held = -1;                 // a claimed target waiting for its parent
  unsigned ticket = kTwNoTicket; // this warp's slot in the continuation queue
  uint32_t idle = 0;
  unsigned backoff = 256;  // ns, doubled while there is nothing to do

  while (true) {
    // ---- fetch.  Each warp holds one queue ticket (taken with a plain
    // atomicAdd, so claims never retry) and runs the piece that lands in its
    // slot; otherwise the held target once its parent is done; otherwise it
    // claims the next target in level order.
    int kind = 0;  // 0 none, 1 piece, 2 target
    TwPiece pc;
    pc.t = -1;
    pc.spill_off = 0;
    pc.spill_cnt = 0;
    pc.inh_b = pc.inh_e = 0;
    if (ticket == kTwNoTicket) {
      unsigned h = 0;
      if (lane == 0) h = atomicAdd(&a.ctl->q_head, 1u);
      ticket = __shfl_sync(0xffffffffu, h, 0);
    }
    if (ticket < a.q_cap) {
      unsigned r = 0;
      if (lane == 0) r = ld_volatile_u32_(&a.q_ready[ticket]);
      r = __shfl_sync(0xffffffffu, r, 0);
      if (r) {
        __threadfence();
        __syncwarp();
        pc = a.queue[ticket];
        ticket = kTwNoTicket;
        kind = 1;
      }
    }
    if (kind == 0 && held >= 0) {
      int ready = 0;
      if (lane == 0) ready = ld_acquire_i32(&a.done[a.parent[held]]);
      ready = __shfl_sync(0xffffffffu, ready, 0);
      __syncwarp();
      if (ready) {
        pc.t = held;
        held = -1;
        kind = 2;
      }
    }
    if (kind == 0 && held < 0) {
      int idx = -1;
      if (lane == 0) {
        if (ld_volatile_u32_(&a.ctl->tick) < (unsigned)a.n_targets) {
          atomicAdd(&a.ctl->work, 1);
          const unsigned i = atomicAdd(&a.ctl->tick, 1u);
          if (i < (unsigned)a.n_targets) idx = (int)i;
          else atomicSub(&a.ctl->work, 1);
        }
      }
      idx = __shfl_sync(0xffffffffu, idx, 0);
      if (idx >= 0) {
        held = a.nbl[a.lo + idx];
        idle = 0;
        backoff = 256;
        continue;  // check its parent next round (queue slot first)
      }
    }
    if (kind == 0) {
      // done when every target is claimed and nothing is outstanding: no
      // piece can be pushed any more (an unfilled ticket is abandoned)
      int fin = 0;
      if (lane == 0)
        fin = held < 0 && ld_volatile_u32_(&a.ctl->tick) >= (unsigned)a.n_targets &&
              ld_volatile_i32_(&a.ctl->work) <= 0;
      fin = __shfl_sync(0xffffffffu, fin, 0);
      if (fin) break;
      __nanosleep(backoff);
      backoff = backoff < 4096 ? backoff * 2 : 4096;
      if (++idle >= a.spin_limit) {
        if (lane == 0) raise_flag(a.status, kFlagTimeout);
        break;
      }
      continue;
    }
    idle = 0;
    backoff = 256;
    if (lane == 0) {
      const long long now = clock64();
      W.st.idle += (unsigned long long)(now - W.t_mark);
      W.t_mark = now;
      W.st.pieces += 1ull;
    }

    // ---- one piece of target t
    const int t = pc.t;
    const float4 Tc = a.recs[t].c;
    const int t_left = a.recs[t].k.x, t_first = a.recs[t].k.w;
    const bool t_leaf = t_left < 0;
    const int p = a.parent[t];
    const int4 pk = a.recs[p].k;  // children of p
    const int sib = pk.x == t ? pk.y : pk.x;
    const int sib_gen = a.level[p] + 1;
    if (kind == 2) {
      pc.spill_cnt = 0;
      pc.inh_b = 0;
      pc.inh_e = a.s_cnt[p] + 1;  // parent's split list plus the sibling
      if (lane == 0) a.pieces_left[t] = 1;
    }
    const long long s_base = a.s_off[p];
    const int s_ins = kOrd ? a.s_ins[p] : 0;
    const int src_len = pc.spill_cnt + (pc.inh_e - pc.inh_b);
    int cur = 0, stk_n = 0, steps = 0, lanes = 0;
    int n_fi = 0, n_fl = 0, n_n = 0, n_s = 0;
    unsigned c_acc = 0, c_near = 0, c_ref = 0;  // this lane's decisions in this piece
    // far rows are keyed by level-major rank (ordered: the chunk sort
    // places them) or by node id (unordered: offset tables per node)
    auto flush_fi = [&]() {
      const unsigned long long hi = (unsigned long long)(uint32_t)(kOrd ? a.rank[t] : t) << 32;
      const bool in_place = !kOrd && a.far_rcap != nullptr;
      tw_flush_rows<kOrd>(W.stg_fi, n_fi, lane, t, hi, 0u, a.far_pool, a.far_cap, &a.ctl->far_cur,
                    &al.far, a.far_keys, a.far_recs, a.far_rec_cap, &a.ctl->far_rec_cur,
                    &al.far_r, &a.far_cnt[t], in_place ? a.far_raw : nullptr,
                    in_place ? a.far_rcap[t] : 0, in_place ? a.pad_far[t] : 0,
                    in_place ? &a.first_ovf_far[t] : nullptr, a);
      n_fi = 0;
    };
    auto flush_fl = [&]() {
      const unsigned long long hi = (unsigned long long)(uint32_t)a.rank[t] << 32;
      tw_flush_rows<kOrd>(W.stg_fl, n_fl, lane, t, hi, 0x80000000u, a.far_pool, a.far_cap,
                    &a.ctl->far_cur, &al.far, a.far_keys, a.far_recs, a.far_rec_cap,
                    &a.ctl->far_rec_cur, &al.far_r, &a.far_cnt[t], nullptr, 0, 0, nullptr, a);
      n_fl = 0;
    };
    auto flush_n = [&]() {
      const int lp = a.recs[t].k.z;  // leaf position (leaf targets only)
      const unsigned long long hi = (unsigned long long)(uint32_t)lp << 32;
      const bool in_place = !kOrd && a.near_rcap != nullptr;
      tw_flush_rows<kOrd>(W.stg_n, n_n, lane, t, hi, 0u, a.near_pool, a.near_cap, &a.ctl->near_cur,
                    &al.near_, a.near_keys, a.near_recs, a.near_rec_cap, &a.ctl->near_rec_cur,
                    &al.near_r, &a.near_cnt[lp], in_place ? a.near_raw : nullptr,
                    in_place ? a.near_rcap[lp] : 0, in_place ? a.pad_near[lp] : 0,
                    in_place ? &a.first_ovf_near[lp] : nullptr, a);
      n_n = 0;
    };
    auto flush_s = [&]() {
      tw_flush_split(W.stg_s, n_s, lane, t, a, al);
      n_s = 0;
    };
    // Pops the next window -- the leftmost (up to) 32 candidates: stack top
    // first, then source -- and requests the node records of its pending
    // candidates (an id outside the tree is not read; it is reported when
    // the window is evaluated).
    auto load_window = [&](unsigned long long& e, int& n, float4& Bc, int4& Bk) {
      const int take_stk = stk_n < 32 ? stk_n : 32;
      const int rest = src_len - cur;
      const int take_src = (32 - take_stk) < rest ? (32 - take_stk) : rest;
      n = take_stk + take_src;
      e = 0ull;
      if (lane < take_stk) {
        e = W.stk[stk_n - 1 - lane];
      } else if (lane < n) {
        const int c = cur + (lane - take_stk);
        if (c < pc.spill_cnt) {
          e = a.spill[pc.spill_off + c];
        } else {
          const int q = pc.inh_b + (c - pc.spill_cnt);
          if (q < s_ins) e = a.s_pool[s_base + q];
          else if (q == s_ins) e = tw_ent(sib, sib_gen, 0, 0);
          else e = a.s_pool[s_base + q - 1];
        }
      }
      stk_n -= take_stk;
      cur += take_src;
      Bc = make_float4(0.f, 0.f, 0.f, 0.f);
      Bk = make_int4(-1, -1, -1, -1);
      if (lane < n && tw_state(e) == 0 && (unsigned)tw_s(e) < (unsigned)a.total) {
        const TwRec* r = a.recs + tw_s(e);
        Bc = r->c;
        Bk = r->k;
      }
      __syncwarp();  // the popped slots are rewritten by later pushes
    };

    unsigned long long e;
    int n;
    float4 Bc;
    int4 Bk;
    load_window(e, n, Bc, Bk);
    while (n > 0) {
      // ---- evaluate pending candidates (an id outside the tree is dropped
      // and reported, never dereferenced)
      bool valid = lane < n;
      if (valid && (unsigned)tw_s(e) >= (unsigned)a.total) {
        raise_flag(a.status, kFlagBadInput);
        valid = false;
      }
      int state = valid ? tw_state(e) : 0;
      bool refine_s = false;
      unsigned long long c0 = 0, c1 = 0;
      if (valid && state == 0) {
        const int s = tw_s(e);
        const int g = tw_gen(e);
        const float dx = __fsub_rn(Tc.x, Bc.x);
        const float dy = __fsub_rn(Tc.y, Bc.y);
        const float dz = __fsub_rn(Tc.z, Bc.z);
        float d2 = __fmul_rn(dx, dx);
        d2 = __fadd_rn(d2, __fmul_rn(dy, dy));
        d2 = __fadd_rn(d2, __fmul_rn(dz, dz));
        const float et = Tc.w, es = Bc.w;
        bool ok;
        if (kMac == kTwEngblom) {
          const float big = fmax_nan(et, es), small = fmin_nan(et, es);
          const float lhs = __fadd_rn(big, __fmul_rn(a.theta, small));
          ok = __fmul_rn(lhs, lhs) <= __fmul_rn(a.theta_sq, d2);
        } else {
          const float sum = __fadd_rn(et, es);
          ok = __fmul_rn(sum, sum) <= __fmul_rn(a.theta_sq, d2);
        }
        const bool s_leaf = Bk.x < 0;
        atomicAdd(&sm.hist[g < kTwHist ? g : kTwHist - 1], 1u);
        if (d2 > 0.0f && ok) {
          state = 1;
          ++c_acc;
        } else if (t_leaf && s_leaf) {
          state = 2;
          ++c_near;
        } else {
          ++c_ref;
          // split rule on the canonical (lo, hi) orientation
          const bool t_lo = t < s;
          const float e_lo = t_lo ? et : es, e_hi = t_lo ? es : et;
          const bool lo_int = t_lo ? !t_leaf : !s_leaf, hi_leaf = t_lo ? s_leaf : t_leaf;
          const bool split_lo = lo_int && (hi_leaf || e_lo >= e_hi);
          const bool split_t = t_lo ? split_lo : !split_lo;
          if (split_t) {
            state = 3;
            e = tw_ent(s, g + 1, 3, (kOrd && Bk.w < t_first) ? 1 : 0);
          } else {
            refine_s = true;
            c0 = tw_ent(Bk.x, g + 1, 0, 0);
            c1 = tw_ent(Bk.y, g + 1, 0, 0);
          }
        }
        if (state == 1 || state == 2) e = tw_ent(s, g, state, 0);
      }
      const unsigned refm = __ballot_sync(0xffffffffu, refine_s);
      // ordered: lanes [0, f) are resolved -- emit them; unordered: every
      // resolved lane
      const int f = kOrd ? (refm ? __ffs(refm) - 1 : n) : n;
      const bool emit = valid && lane < f && (kOrd || !refine_s);
      // ---- stage this window's emitted entries (flushing when full)
      auto emit_window = [&]() {
        const int s = tw_s(e);
        const bool is_fi = emit && state == 1 && (!kOrd || s < a.ni);
        const bool is_fl = kOrd && emit && state == 1 && s >= a.ni;
        const bool is_n = emit && state == 2;
        const bool is_s = emit && state == 3;
        const unsigned mfi = __ballot_sync(0xffffffffu, is_fi);
        const unsigned mfl = kOrd ? __ballot_sync(0xffffffffu, is_fl) : 0u;
        const unsigned mn = __ballot_sync(0xffffffffu, is_n);
        const unsigned ms = __ballot_sync(0xffffffffu, is_s);
        if (mfi) {
          if (n_fi + __popc(mfi) > kTwStgF) {
            __syncwarp();
            flush_fi();
            __syncwarp();
          }
          if (is_fi) W.stg_fi[n_fi + __popc(mfi & lt)] = s;
          n_fi += __popc(mfi);
        }
        if (kOrd && mfl) {
          if (n_fl + __popc(mfl) > kTwStgF) {
            __syncwarp();
            flush_fl();
            __syncwarp();
          }
          if (is_fl) W.stg_fl[n_fl + __popc(mfl & lt)] = s;
          n_fl += __popc(mfl);
        }
        if (mn) {
          if (n_n + __popc(mn) > kTwStgF) {
            __syncwarp();
            flush_n();
            __syncwarp();
          }
          if (is_n) W.stg_n[n_n + __popc(mn & lt)] = s;
          n_n += __popc(mn);
        }
        if (ms) {
          if (n_s + __popc(ms) > kTwStgS) {
            __syncwarp();
            flush_s();
            __syncwarp();
          }
          if (is_s) W.stg_s[n_s + __popc(ms & lt)] = e;
          n_s += __popc(ms);
        }
      };
      // ---- outputs that go back on the stack: ordered, lanes [f, n) in
      // order (children replace their parent); unordered, the children
      int nout, P, k0;  // this lane's outputs, the warp's, this lane's first index
      if (kOrd) {
        nout = (valid && lane >= f) ? (refine_s ? 2 : 1) : 0;
        int incl = nout;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        P = __shfl_sync(0xffffffffu, incl, 31);
        k0 = incl - nout;
      } else {
        nout = refine_s ? 2 : 0;
        P = 2 * __popc(refm);
        k0 = 2 * __popc(refm & lt);
      }
      ++steps;
      lanes += n;
      if (stk_n + P > kTwStk) {
        // no room on the stack: hand these outputs, the stack and the rest
        // of the source to other warps
        emit_window();
        tw_hand_off(a, lane, t, pc, cur, nout, k0, refine_s ? c0 : e, c1, P, W.stk, stk_n);
        stk_n = 0;
        cur = src_len;
        break;
      }
      if (nout >= 1) W.stk[stk_n + P - 1 - k0] = refine_s ? c0 : e;
      if (nout == 2) W.stk[stk_n + P - 2 - k0] = c1;
      stk_n += P;
      __syncwarp();
      if (steps >= a.budget && (stk_n > 0 || cur < src_len)) {
        // out of budget: hand the stack and the rest of the source off
        emit_window();
        tw_hand_off(a, lane, t, pc, cur, 0, 0, 0ull, 0ull, 0, W.stk, stk_n);
        stk_n = 0;
        cur = src_len;
        break;
      }
      // ---- next window first (its record gathers are in flight while this
      // window's entries are staged), then this window's emission
      unsigned long long e2;
      int n2;
      float4 Bc2;
      int4 Bk2;
      load_window(e2, n2, Bc2, Bk2);
      emit_window();
      e = e2;
      n = n2;
      Bc = Bc2;
      Bk = Bk2;
    }
    // ---- end of the piece: flush, then account
    __syncwarp();
    flush_fi();
    if (kOrd) flush_fl();
    if (t_leaf) flush_n();
    flush_s();
    for (int o = 16; o > 0; o >>= 1) {
      c_acc += __shfl_xor_sync(0xffffffffu, c_acc, o);
      c_near += __shfl_xor_sync(0xffffffffu, c_near, o);
      c_ref += __shfl_xor_sync(0xffffffffu, c_ref, o);
    }
    if (lane == 0) {
      W.st.acc += c_acc;
      W.st.near_ += c_near;
      W.st.ref += c_ref;
      W.st.steps += (unsigned long long)steps;
      W.st.lanes += (unsigned long long)lanes;
    }
    __syncwarp();
    int last = 0;
    if (lane == 0) {
      __threadfence();
      last = atomicSub(&a.pieces_left[t], 1) == 1;
      if (last) __threadfence();
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
      if (!t_leaf) tw_compact_split<kOrd>(t, lane, a, W.stk);
      __syncwarp();
      if (lane == 0) {
        __threadfence();
        st_release_i32(&a.done[t], 1);
      }
    }
    if (lane == 0) {
      atomicSub(&a.ctl->work, 1);
      const long long now = clock64();
      W.st.busy += (unsigned long long)(now - W.t_mark);
      W.t_mark = now;
    }
    __syncwarp();
  }
  // ---- unused record slots of this warp's last blocks: empty chunks
  __syncwarp();
  for (unsigned long long k = al.far_r.cur + lane; k < al.far_r.end; k += 32) {
    a.far_keys[k] = 0ull;
    TwChunk c;
    c.off = 0;
    c.cnt = 0;
    c.t = 0;
    a.far_recs[k] = c;
  }
  for (unsigned long long k = al.near_r.cur + lane; k < al.near_r.end; k += 32) {
    a.near_keys[k] = 0ull;
    TwChunk c;
    c.off = 0;
    c.cnt = 0;
    c.t = 0;
    a.near_recs[k] = c;
  }
  // ---- statistics
  if (lane == 0) {
    W.st.idle += (unsigned long long)(clock64() - W.t_mark);
    const TwWarpStats& q = W.st;
    if (q.acc) atomicAdd(&a.ctl->acc_sides, q.acc);
    if (q.near_) atomicAdd(&a.ctl->near_sides, q.near_);
    if (q.ref) atomicAdd(&a.ctl->ref_sides, q.ref);
    atomicAdd(&a.ctl->busy_cycles, q.busy);
    atomicAdd(&a.ctl->idle_cycles, q.idle);
    atomicAdd(&a.ctl->pieces, q.pieces);
    atomicAdd(&a.ctl->steps, q.steps);
    atomicAdd(&a.ctl->lanes, q.lanes);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kTwHist; i += kTwThreads)
    if (sm.hist[i]) atomicAdd(&a.gen_hist[i], sm.hist[i]);
}

// ---------------------------------------------------------------------------
// statistics and assembly

// Row totals and maxima (far per node, near per leaf position).
__global__ void k_tw_row_stats(const int32_t* __restrict__ far_cnt, int32_t total,
                               const int32_t* __restrict__ near_cnt, int32_t L,
                               unsigned long long* __restrict__ out) {
  unsigned long long fs = 0, ns = 0, fm = 0, nm = 0;
  for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    const unsigned long long v = (unsigned long long)far_cnt[k];
    fs += v;
    fm = v > fm ? v : fm;
    if (k < L) {
      const unsigned long long w = (unsigned long long)near_cnt[k];
      ns += w;
      nm = w > nm ? w : nm;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    fs += __shfl_xor_sync(0xffffffffu, fs, o);
    ns += __shfl_xor_sync(0xffffffffu, ns, o);
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, fm, o);
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, nm, o);
    fm = x > fm ? x : fm;
    nm = y > nm ? y : nm;
  }
  if ((threadIdx.x & 31) == 0) {
    if (fs) atomicAdd(&out[0], fs);
    if (ns) atomicAdd(&out[1], ns);
    atomicMax(&out[2], fm);
    atomicMax(&out[3], nm);
  }
}

// Chunk counts in sorted key order.
__global__ void k_tw_sorted_counts(const uint32_t* __restrict__ order, const TwChunk* __restrict__ recs,
                                   int64_t m, int32_t* __restrict__ cnt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x)
    cnt[i] = recs[order[i]].cnt;
}

// One warp per chunk (in sorted order): copies its entries to their final
// place, widened to the index dtype; far chunks also write the target and
// its level for every entry.
__global__ void __launch_bounds__(256)
    k_tw_copy(const uint32_t* __restrict__ order, const TwChunk* __restrict__ recs, int64_t m,
              const int64_t* __restrict__ dest, const int32_t* __restrict__ pool, int index_bits,
              void* vals_out, void* tgt_out, void* lvl_out, const int32_t* __restrict__ level) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = w0; i < m; i += nw) {
    const TwChunk c = recs[order[i]];
    const int64_t d = dest[i];
    const int lv = tgt_out ? level[c.t] : 0;
    for (int k = lane; k < c.cnt; k += 32) {
      store_idx(vals_out, index_bits, d + k, pool[c.off + k]);
      if (tgt_out) {
        store_idx(tgt_out, index_bits, d + k, c.t);
        store_idx(lvl_out, index_bits, d + k, lv);
      }
    }
  }
}

// Unordered rows: one warp per chunk record (any order) copies the chunk's
// entries to the row's raw area at base[row] + the chunk's offset within
// the row (record key: row << 32 | offset); the rows are sorted afterwards.
// A record that does not fit its row or its pool is reported, not copied.
__global__ void __launch_bounds__(256)
    k_tw_copy_raw(const unsigned long long* __restrict__ keys, const TwChunk* __restrict__ recs,
                  int64_t m, const int64_t* __restrict__ base, int64_t rows,
                  const int32_t* __restrict__ pool, int64_t pool_cap, int32_t* __restrict__ raw,
                  int64_t raw_cap, uint32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = w0; i < m; i += nw) {
    const TwChunk c = recs[i];
    if (c.cnt <= 0) continue;
    const unsigned long long k = keys[i];
    if ((int64_t)(k >> 32) >= rows || c.off < 0 || c.off + c.cnt > pool_cap) {
      if (lane == 0) raise_flag(status, kFlagMalformed);
      continue;
    }
    const int64_t d = base[k >> 32] + (int64_t)(k & 0xffffffffull);
    if (d < 0 || d + c.cnt > raw_cap) {
      if (lane == 0) raise_flag(status, kFlagMalformed);
      continue;
    }
    for (int e = lane; e < c.cnt; e += 32) raw[d + e] = pool[c.off + e];
  }
}

// Predicted rows: per list, the rows that outgrew their capacity, the
// entries past the capacities and the entries those rows hold (their
// extension).  out: ovf rows, ovf entries, far extension, near extension.
__global__ void k_tw_ext_stats(const int32_t* __restrict__ far_cnt,
                               const int32_t* __restrict__ far_rcap, int32_t total,
                               const int32_t* __restrict__ near_cnt,
                               const int32_t* __restrict__ near_rcap, int32_t L,
                               unsigned long long* __restrict__ out) {
  unsigned long long rows = 0, past = 0, ef = 0, en = 0;
  for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    const int32_t c = far_cnt[k], r = far_rcap[k];
    if (c > r) {
      ++rows;
      past += (unsigned long long)(c - r);
      ef += (unsigned long long)c;
    }
    if (k < L) {
      const int32_t cn = near_cnt[k], rn = near_rcap[k];
      if (cn > rn) {
        ++rows;
        past += (unsigned long long)(cn - rn);
        en += (unsigned long long)cn;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    rows += __shfl_xor_sync(0xffffffffu, rows, o);
    past += __shfl_xor_sync(0xffffffffu, past, o);
    ef += __shfl_xor_sync(0xffffffffu, ef, o);
    en += __shfl_xor_sync(0xffffffffu, en, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (rows) atomicAdd(&out[0], rows);
    if (past) atomicAdd(&out[1], past);
    if (ef) atomicAdd(&out[2], ef);
    if (en) atomicAdd(&out[3], en);
  }
}

// Extension length of every row: its count if it outgrew the capacity.
__global__ void k_tw_ext_len(const int32_t* __restrict__ cnt, const int32_t* __restrict__ rcap,
                             int32_t rows, int32_t* __restrict__ ext_len) {
  for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < rows; k += gridDim.x * blockDim.x)
    ext_len[k] = cnt[k] > rcap[k] ? cnt[k] : 0;
}

// Where every row's raw entries sit: its padded slot, or for a row that
// outgrew it, its extension behind all padded slots.
__global__ void k_tw_roff(const int32_t* __restrict__ cnt, const int32_t* __restrict__ rcap,
                          const int64_t* __restrict__ pad, const int64_t* __restrict__ ext_off,
                          int32_t rows, int64_t* __restrict__ roff) {
  const int64_t pad_total = pad[rows];
  for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < rows; k += gridDim.x * blockDim.x)
    roff[k] = cnt[k] > rcap[k] ? pad_total + ext_off[k] : pad[k];
}

// A row that outgrew its slot: the entries written in place (offsets below
// the first one that went to the pool) move to the front of its extension.
// The extensions lie back to back behind all slots (ext_off: exclusive sums
// of the rows' extension lengths, rows + 1 entries), so the copy runs over
// blocks of 1024 extension positions, one warp per block, each finding its
// rows by binary search: a halo row of 10^5 entries is spread over many
// warps instead of one.
__device__ __forceinline__ int32_t tw_row_of(const int64_t* __restrict__ ext_off, int32_t rows,
                                             int64_t x) {
  // last r with ext_off[r] <= x (its extension then holds x)
  int32_t lo = 0, hi = rows;  // ext_off[0] = 0 <= x < ext_off[rows]
  while (hi - lo > 1) {
    const int32_t mid = (lo + hi) >> 1;
    if (ext_off[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}
__global__ void k_tw_prefix_copy(const int32_t* __restrict__ cnt, const int64_t* __restrict__ pad,
                                 const unsigned* __restrict__ first_ovf,
                                 const int64_t* __restrict__ ext_off, int32_t rows,
                                 int32_t* __restrict__ raw, int64_t raw_cap,
                                 uint32_t* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ext_total = ext_off[rows], pad_total = pad[rows];
  if (pad_total + ext_total > raw_cap) {  // reported, nothing copied
    if (w0 == 0 && lane == 0) raise_flag(status, kFlagMalformed);
    return;
  }
  for (int64_t x0 = w0 * 1024; x0 < ext_total; x0 += nw * 1024) {
    const int64_t x1 = x0 + 1024 < ext_total ? x0 + 1024 : ext_total;
    int64_t x = x0;
    while (x < x1) {
      const int32_t r = tw_row_of(ext_off, rows, x);
      const int64_t rb = ext_off[r], re = ext_off[r + 1];
      const int64_t seg_end = re < x1 ? re : x1;
      const unsigned fo = first_ovf[r];
      const int64_t P = fo < (unsigned)cnt[r] ? (int64_t)fo : (int64_t)cnt[r];
      const int64_t src = pad[r];
      for (int64_t xx = x + lane; xx < seg_end; xx += 32) {
        const int64_t k = xx - rb;
        if (k < P) raw[pad_total + xx] = raw[src + k];
      }
      x = seg_end > x ? seg_end : x1;  // a zero-length row cannot hold x
    }
  }
}

// counts in nodes_by_level order; far offsets; index-dtype tables
__global__ void k_tw_gather(const int32_t* __restrict__ cnt, const int32_t* __restrict__ nbl,
                            int32_t m, int32_t* __restrict__ out) {
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
    out[r] = cnt[nbl[r]];
}
__global__ void k_tw_far_tables(const int64_t* __restrict__ obl, const int32_t* __restrict__ nbl,
                                const int32_t* __restrict__ cnt, int32_t total, int index_bits,
                                void* node_offsets, void* counts_out, const void* tree_level_offsets,
                                int num_levels, void* level_offsets_out,
                                int64_t* __restrict__ off_node) {
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= total; r += gridDim.x * blockDim.x) {
    if (r == total) {
      store_idx(node_offsets, index_bits, total, obl[total]);
      if (off_node) off_node[total] = obl[total];
    } else {
      const int32_t v = nbl[r];
      store_idx(node_offsets, index_bits, v, obl[r]);
      if (off_node) off_node[v] = obl[r];
      store_idx(counts_out, index_bits, v, cnt[v]);
    }
    if (r <= num_levels) {
      const int64_t li = load_idx(tree_level_offsets, index_bits, r);
      store_idx(level_offsets_out, index_bits, r, obl[li]);
    }
  }
}
__global__ void k_tw_near_tables(const int64_t* __restrict__ off, const int32_t* __restrict__ cnt,
                                 int32_t L, int index_bits, void* offsets_out, void* counts_out) {
  for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j <= L; j += gridDim.x * blockDim.x) {
    store_idx(offsets_out, index_bits, j, off[j]);
    if (j < L) store_idx(counts_out, index_bits, j, cnt[j]);
  }
}

// Dense neighbour leaf positions (L x max_nbr, -1 padded) of
// _result_to_neighbors (:3658-3688).
__global__ void k_tw_nbr_leaf_pos(const int64_t* __restrict__ near_off,
                                  const int32_t* __restrict__ near_cnt, int64_t L,
                                  const void* neighbors, int index_bits,
                                  const int32_t* __restrict__ leafpos, int64_t max_nbr, void* out) {
  const int64_t n = L * max_nbr;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / max_nbr, k = e - j * max_nbr;
    int64_t v = -1;
    if (k < near_cnt[j]) v = leafpos[load_idx(neighbors, index_bits, near_off[j] + k)];
    store_idx(out, index_bits, e, v);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// workspace

struct TwCaps {
  int64_t far, near_, split, spill, far_rec, near_rec, s_rec, queue;
};

struct TwScratch {
  uint32_t* status;
  TwCtl* ctl;
  unsigned int* gen_hist;
  unsigned long long* rowstat;  // 4 words
  TwRec* recs;
  int32_t* first;
  int32_t* rank;
  long long* s_off;
  int32_t* s_cnt;
  int32_t* s_ins;
  int32_t* s_head;
  int32_t* s_nch;
  int32_t* pieces_left;
  int32_t* done;
  int32_t* far_cnt;
  int32_t* near_cnt;
  int32_t* far_pool;
  int32_t* near_pool;
  unsigned long long* s_pool;
  unsigned long long* spill;
  unsigned long long* far_keys;
  TwChunk* far_recs;
  unsigned long long* near_keys;
  TwChunk* near_recs;
  TwSChunk* s_recs;
  TwPiece* queue;
  unsigned int* q_ready;
  // assembly
  uint32_t* order;            // sorted record indices (max of far / near records)
  unsigned long long* keys_sorted;
  int32_t* sorted_cnt;
  int64_t* dest;
  int64_t* scan_tmp;
  int32_t* cnt_by_level;
  int64_t* obl;
  int64_t* near_off;
  void* sort_ws;
  size_t sort_ws_bytes;
  // unordered walks: rows assembled raw (caller's arrays), then sorted
  int64_t* far_off_node;
  unsigned* first_ovf_far;  // predicted rows
  unsigned* first_ovf_near;
  int32_t* ext_len;
  int64_t* ext_off;
  int64_t* roff_far;
  int64_t* roff_near;
  RowSortScratch rs;
};

static TwScratch carve_tw(Arena& a, int64_t total, int64_t L, const TwCaps& c, bool ordered) {
  TwScratch s;
  // status word, control block, histogram and row stats first: one memset
  s.status = a.take<uint32_t>(64);
  s.ctl = a.take<TwCtl>(1);
  s.gen_hist = a.take<unsigned int>(kTwHist);
  s.rowstat = a.take<unsigned long long>(8);
  // per node, zeroed: split counts, insertion points, chunk counts, pieces
  s.s_cnt = a.take<int32_t>(total);
  s.s_ins = a.take<int32_t>(total);
  s.s_nch = a.take<int32_t>(total);
  s.pieces_left = a.take<int32_t>(total);
  s.far_cnt = a.take<int32_t>(total);
  s.near_cnt = a.take<int32_t>(L > 0 ? L : 1);
  // per node, written before use
  s.recs = a.take<TwRec>(total);
  s.first = a.take<int32_t>(total);
  s.rank = a.take<int32_t>(total);
  s.s_off = a.take<long long>(total);
  s.s_head = a.take<int32_t>(total);
  s.done = a.take<int32_t>(total);
  s.q_ready = a.take<unsigned int>(c.queue);
  s.far_pool = a.take<int32_t>(c.far);
  s.near_pool = a.take<int32_t>(c.near_);
  s.s_pool = a.take<unsigned long long>(c.split);
  s.spill = a.take<unsigned long long>(c.spill);
  s.far_keys = a.take<unsigned long long>(c.far_rec);
  s.far_recs = a.take<TwChunk>(c.far_rec);
  s.near_keys = a.take<unsigned long long>(c.near_rec);
  s.near_recs = a.take<TwChunk>(c.near_rec);
  s.s_recs = a.take<TwSChunk>(c.s_rec);
  s.queue = a.take<TwPiece>(c.queue);
  const int64_t mrec = c.far_rec > c.near_rec ? c.far_rec : c.near_rec;
  s.order = a.take<uint32_t>(mrec);
  s.keys_sorted = a.take<unsigned long long>(mrec);
  s.sorted_cnt = a.take<int32_t>(mrec);
  s.dest = a.take<int64_t>(mrec + 1);
  const int64_t scan_n = mrec > total ? mrec : total;
  s.scan_tmp = a.take<int64_t>(scan_scratch_elems(scan_n));
  s.cnt_by_level = a.take<int32_t>(total);
  s.obl = a.take<int64_t>(total + 1);
  s.near_off = a.take<int64_t>((L > 0 ? L : 1) + 1);
  s.sort_ws_bytes = onesweep_scratch_bytes(mrec) + 256;
  s.sort_ws = a.take<unsigned char>(s.sort_ws_bytes);
  s.far_off_node = nullptr;
  s.first_ovf_far = s.first_ovf_near = nullptr;
  s.ext_len = nullptr;
  s.ext_off = s.roff_far = s.roff_near = nullptr;
  s.rs = RowSortScratch{nullptr, nullptr, nullptr, nullptr, 0};
  if (!ordered) {
    const int64_t mx = (total > L ? total : L) + 1;
    s.far_off_node = a.take<int64_t>(total + 1);
    s.first_ovf_far = a.take<unsigned>(total);
    s.first_ovf_near = a.take<unsigned>(L > 0 ? L : 1);
    s.ext_len = a.take<int32_t>(mx);
    s.ext_off = a.take<int64_t>(mx);
    s.roff_far = a.take<int64_t>(total);
    s.roff_near = a.take<int64_t>(L > 0 ? L : 1);
    s.rs = carve_row_sort(a, total, L);
  }
  return s;
}

static bool caps_ok(const TwCaps& c) {
  return c.far >= 1 && c.near_ >= 1 && c.split >= 1 && c.spill >= 1 && c.far_rec >= 1 &&
         c.near_rec >= 1 && c.s_rec >= 1 && c.queue >= 1 && c.far_rec < (int64_t)UINT32_MAX &&
         c.near_rec < (int64_t)UINT32_MAX && c.s_rec < (int64_t)INT32_MAX &&
         c.queue < (int64_t)UINT32_MAX && c.far_rec < (1ll << 30) && c.near_rec < (1ll << 30);
}

}  // namespace ygx

extern "C" {

size_t ygx_target_walk_workspace_size(int64_t total, int64_t num_leaves, const int64_t* caps,
                                      int ordered) {
  if (!caps) return 0;
  ygx::TwCaps c{caps[0], caps[1], caps[2], caps[3], caps[4], caps[5], caps[6], caps[7]};
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_tw(a, total, num_leaves, c, ordered != 0);
  return a.used + 256;
}

int ygx_target_walk(const float* center, const float* radius, const float* max_extent,
                    const int32_t* left32, const int32_t* right32, const int32_t* leafpos32,
                    const int32_t* parent32, const int32_t* level32, const int32_t* nbl32,
                    int64_t total, int64_t num_internal, int root, int mac, float theta,
                    float dehnen_radius_scale, const int64_t* caps, int ordered,
                    const int32_t* far_rcap32, const int32_t* near_rcap32,
                    const int64_t* pad_far, const int64_t* pad_near, int32_t* far_raw,
                    int32_t* near_raw, const void* tree_level_offsets, int num_levels,
                    int index_bits, uint64_t* stats_out, uint64_t* needs_out,
                    uint32_t* flags_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
  using namespace ygx;
  if (total < 3 || total > INT32_MAX || num_internal < 1 || mac < 0 || mac > 2 || !caps ||
      !stats_out || !needs_out || !flags_out || !tree_level_offsets || num_levels < 2 ||
      num_levels > kTwHist / 2 || root < 0 || root >= total ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  if (!center || !radius || !max_extent || !left32 || !right32 || !leafpos32 || !parent32 ||
      !level32 || !nbl32 || !ws)
    return YGX_ERR_ARG;
  const bool pred = far_rcap32 != nullptr;
  if (pred && (ordered || !near_rcap32 || !pad_far || !pad_near || !far_raw || !near_raw))
    return YGX_ERR_ARG;
  if (!pred && (near_rcap32 || pad_far || pad_near || far_raw || near_raw)) return YGX_ERR_ARG;
  TwCaps c{caps[0], caps[1], caps[2], caps[3], caps[4], caps[5], caps[6], caps[7]};
  if (!caps_ok(c)) return YGX_ERR_ARG;
  if (ws_bytes < ygx_target_walk_workspace_size(total, total - num_internal, caps, ordered))
    return YGX_ERR_ARG;
  const int64_t L = total - num_internal;
  Arena ar{(char*)ws, 0, ws_bytes};
  TwScratch s = carve_tw(ar, total, L, c, ordered != 0);
  const size_t zero_bytes = (size_t)((char*)(s.near_cnt + (L > 0 ? L : 1)) - (char*)s.status);
  if (cudaMemsetAsync(s.status, 0, zero_bytes, stream) != cudaSuccess ||
      cudaMemsetAsync(s.q_ready, 0, sizeof(unsigned int) * c.queue, stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  if (pred && (cudaMemsetAsync(s.first_ovf_far, 0xff, sizeof(unsigned) * total, stream) !=
                   cudaSuccess ||
               cudaMemsetAsync(s.first_ovf_near, 0xff, sizeof(unsigned) * (L > 0 ? L : 1),
                               stream) != cudaSuccess))
    return YGX_ERR_CUDA;
  const int32_t T = (int32_t)total, NI = (int32_t)num_internal;
  k_tw_first_leaf<<<grid_for(L, 256), 256, 0, stream>>>(parent32, left32, NI, T, s.first);
  YGX_CHECK_LAUNCH();
  k_tw_recs<<<grid_for(total, 256), 256, 0, stream>>>(center, radius, max_extent, left32,
                                                      right32, leafpos32, s.first, T, mac,
                                                      dehnen_radius_scale, nbl32, s.rank, s.recs,
                                                      s.status);
  YGX_CHECK_LAUNCH();
  k_tw_init_nodes<<<grid_for(total, 256), 256, 0, stream>>>(T, root, s.s_head, s.s_off, s.done);
  YGX_CHECK_LAUNCH();
  const float th = theta;
  TwArgs a;
  a.recs = s.recs;
  a.nbl = nbl32;
  a.parent = parent32;
  a.level = level32;
  a.rank = s.rank;
  a.ni = NI;
  a.total = T;
  a.lo = 1;  // level 0 holds the root alone
  a.n_targets = T - 1;
  a.theta_sq = th * th;
  a.theta = sqrtf(a.theta_sq);
  a.s_off = s.s_off;
  a.s_cnt = s.s_cnt;
  a.s_ins = s.s_ins;
  a.s_head = s.s_head;
  a.s_nch = s.s_nch;
  a.pieces_left = s.pieces_left;
  a.done = s.done;
  a.far_cnt = s.far_cnt;
  a.near_cnt = s.near_cnt;
  a.far_pool = s.far_pool;
  a.near_pool = s.near_pool;
  a.s_pool = s.s_pool;
  a.spill = s.spill;
  a.far_cap = (unsigned long long)c.far;
  a.near_cap = (unsigned long long)c.near_;
  a.s_cap = (unsigned long long)c.split;
  a.spill_cap = (unsigned long long)c.spill;
  a.far_keys = s.far_keys;
  a.far_recs = s.far_recs;
  a.near_keys = s.near_keys;
  a.near_recs = s.near_recs;
  a.s_recs = s.s_recs;
  a.far_rec_cap = (unsigned)c.far_rec;
  a.near_rec_cap = (unsigned)c.near_rec;
  a.s_rec_cap = (unsigned)c.s_rec;
  a.q_cap = (unsigned)c.queue;
  a.queue = s.queue;
  a.q_ready = s.q_ready;
  a.gen_hist = s.gen_hist;
  a.ctl = s.ctl;
  a.status = s.status;
  a.spin_limit = (uint32_t)g_tune.spin_limit;
  a.budget = g_tune.target_budget;
  a.far_rcap = pred ? far_rcap32 : nullptr;
  a.near_rcap = pred ? near_rcap32 : nullptr;
  a.pad_far = pad_far;
  a.pad_near = pad_near;
  a.far_raw = far_raw;
  a.near_raw = near_raw;
  a.first_ovf_far = pred ? s.first_ovf_far : nullptr;
  a.first_ovf_near = pred ? s.first_ovf_near : nullptr;
  {
    // allocation blocks: small enough that every warp's open blocks fit the
    // pools many times over, large enough to keep the global cursors quiet
    const long long nwarps = (long long)kNumSMs * kTwBlocksPerSM * kTwWarps;
    long long me = c.far < c.near_ ? c.far : c.near_;
    me = me < c.split ? me : c.split;
    long long be = me / (nwarps * 16);
    a.blk_entries = (unsigned long long)(be < 32 ? 32 : (be > 2048 ? 2048 : be));
    long long mr = c.far_rec < c.near_rec ? c.far_rec : c.near_rec;
    mr = mr < c.s_rec ? mr : c.s_rec;
    long long br = mr / (nwarps * 8);
    a.blk_records = (unsigned)(br < 4 ? 4 : (br > 64 ? 64 : br));
  }
  const size_t smem = sizeof(TwSmem);
  static std::atomic<uint64_t> attr[6];
  const int grid = kNumSMs * kTwBlocksPerSM;
  cudaError_t e = cudaSuccess;
#define YGX_TW(M, O, I)                                                         \
  e = ensure_smem_limit(k_tw_walk<M, O>, (int)smem, attr[I]);                   \
  if (e == cudaSuccess) k_tw_walk<M, O><<<grid, kTwThreads, smem, stream>>>(a);
  if (ordered) {
    switch (mac) {
      case kTwBH: YGX_TW(kTwBH, true, 0) break;
      case kTwDehnen: YGX_TW(kTwDehnen, true, 1) break;
      default: YGX_TW(kTwEngblom, true, 2) break;
    }
  } else {
    switch (mac) {
      case kTwBH: YGX_TW(kTwBH, false, 3) break;
      case kTwDehnen: YGX_TW(kTwDehnen, false, 4) break;
      default: YGX_TW(kTwEngblom, false, 5) break;
    }
  }
#undef YGX_TW
  if (e != cudaSuccess) return YGX_ERR_CUDA;
  YGX_CHECK_LAUNCH();
  k_tw_row_stats<<<grid_for(total, 256, kNumSMs * 4), 256, 0, stream>>>(s.far_cnt, T, s.near_cnt,
                                                                       (int32_t)L, s.rowstat);
  YGX_CHECK_LAUNCH();
  if (pred) {
    k_tw_ext_stats<<<grid_for(total, 256, kNumSMs * 4), 256, 0, stream>>>(
        s.far_cnt, far_rcap32, T, s.near_cnt, near_rcap32, (int32_t)L, s.rowstat + 4);
    YGX_CHECK_LAUNCH();
  }
  TwCtl ctl;
  unsigned int hist[kTwHist];
  unsigned long long rs[8];
  int64_t lvl_off[kTwHist / 2 + 1];
  int32_t lvl_off32[kTwHist / 2 + 1];
  const bool i64 = index_bits == 64;
  if (cudaMemcpyAsync(i64 ? (void*)lvl_off : (void*)lvl_off32, tree_level_offsets,
                      (size_t)(num_levels + 1) * (i64 ? 8 : 4), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaMemcpyAsync(&ctl, s.ctl, sizeof(TwCtl), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(hist, s.gen_hist, sizeof(hist), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(rs, s.rowstat, sizeof(rs), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(flags_out, s.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  // generations: every node's self pair {v, v} sits at generation depth(v);
  // every other pair was evaluated once from each side
  unsigned long long wf2[kTwHist];
  for (int g = 0; g < kTwHist; ++g) wf2[g] = hist[g];
  if (!i64)
    for (int l = 0; l <= num_levels; ++l) lvl_off[l] = lvl_off32[l];
  for (int l = 0; l < num_levels && l < kTwHist; ++l)
    wf2[l] += 2ull * (unsigned long long)(lvl_off[l + 1] - lvl_off[l]);
  unsigned long long mw = 1, gens = 0;
  for (int g = 0; g < kTwHist; ++g) {
    if (wf2[g] == 0) continue;
    gens = (unsigned long long)g + 1;
    if (g > 0 && wf2[g] / 2 > mw) mw = wf2[g] / 2;
  }
  for (int k = 0; k < YGX_TSTAT_WORDS; ++k) stats_out[k] = 0;
  stats_out[YGX_TSTAT_FAR_TOTAL] = rs[0];
  stats_out[YGX_TSTAT_NEAR_TOTAL] = rs[1];
  stats_out[YGX_TSTAT_MAX_FAR] = rs[2];
  stats_out[YGX_TSTAT_MAX_NEAR] = rs[3];
  stats_out[YGX_TSTAT_ACCEPT] = ctl.acc_sides / 2;
  stats_out[YGX_TSTAT_NEAR] = ctl.near_sides / 2;
  stats_out[YGX_TSTAT_REFINE] = ctl.ref_sides / 2 + (unsigned long long)total;
  stats_out[YGX_TSTAT_MAX_WF] = mw;
  stats_out[YGX_TSTAT_GENS] = gens;
  if (pred) {
    stats_out[YGX_TSTAT_OVF_ROWS] = rs[4];
    stats_out[YGX_TSTAT_OVF_ENTRIES] = rs[5];
    stats_out[YGX_TSTAT_EXT_FAR] = rs[6];
    stats_out[YGX_TSTAT_EXT_NEAR] = rs[7];
  }
  // what each capacity needed (a re-run with these fits)
  needs_out[0] = ctl.far_cur;
  needs_out[1] = ctl.near_cur;
  needs_out[2] = ctl.s_cur;
  needs_out[3] = ctl.spill_cur;
  needs_out[4] = ctl.far_rec_cur;
  needs_out[5] = ctl.near_rec_cur;
  needs_out[6] = ctl.s_rec_cur;
  needs_out[7] = ctl.q_tail;
  needs_out[8] = ctl.max_cmp;
  needs_out[9] = ctl.busy_cycles;  // warp cycles on pieces / waiting, pieces run
  needs_out[10] = ctl.idle_cycles;
  needs_out[11] = ctl.pieces;
  needs_out[12] = ctl.steps;  // 32-wide steps and the candidates they held
  needs_out[13] = ctl.lanes;
  return YGX_OK;
}

// After ygx_target_walk on the same workspace (and with its capacities):
// the level-major far lists and the leaf-order near lists in the index dtype,
// with the reference's offset / count tables.
int ygx_target_walk_lists(int64_t total, int64_t num_internal, const int64_t* caps, int ordered,
                          const int32_t* far_rcap32, const int32_t* near_rcap32,
                          const int64_t* pad_far, const int64_t* pad_near, int32_t* far_raw,
                          int64_t far_raw_cap, int32_t* near_raw, int64_t near_raw_cap,
                          const int32_t* nbl32, const int32_t* level32,
                          const void* tree_level_offsets, int num_levels, int index_bits,
                          int64_t far_total, int64_t near_total, uint64_t far_records,
                          uint64_t near_records, void* node_offsets, void* far_counts,
                          void* level_offsets, void* sources, void* targets, void* target_levels,
                          void* near_offsets, void* near_counts, void* neighbors,
                          const int32_t* leafpos32, int64_t max_nbr,
                          void* neighbor_leaf_positions, void* ws, size_t ws_bytes,
                          cudaStream_t stream) {
  using namespace ygx;
  if (total < 3 || num_internal < 1 || !caps || !ws || (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  TwCaps c{caps[0], caps[1], caps[2], caps[3], caps[4], caps[5], caps[6], caps[7]};
  if (!caps_ok(c)) return YGX_ERR_ARG;
  if (ws_bytes < ygx_target_walk_workspace_size(total, total - num_internal, caps, ordered))
    return YGX_ERR_ARG;
  if ((int64_t)far_records > c.far_rec || (int64_t)near_records > c.near_rec) return YGX_ERR_ARG;
  const bool pred = far_rcap32 != nullptr;
  if (ordered && (pred || far_raw || near_raw)) return YGX_ERR_ARG;
  if (!ordered && (!far_raw || !near_raw)) return YGX_ERR_ARG;
  if (pred && (!near_rcap32 || !pad_far || !pad_near)) return YGX_ERR_ARG;
  if (!ordered && !pred && (far_total > far_raw_cap || near_total > near_raw_cap))
    return YGX_ERR_ARG;
  const int64_t L = total - num_internal;
  Arena ar{(char*)ws, 0, ws_bytes};
  TwScratch s = carve_tw(ar, total, L, c, ordered != 0);
  const int32_t T = (int32_t)total;
  // offset / count tables
  k_tw_gather<<<grid_for(total, 256), 256, 0, stream>>>(s.far_cnt, nbl32, T, s.cnt_by_level);
  YGX_CHECK_LAUNCH();
  int rc = exclusive_scan<int32_t>(s.cnt_by_level, total, s.obl, s.scan_tmp, stream);
  if (rc) return rc;
  k_tw_far_tables<<<grid_for(total + 1, 256), 256, 0, stream>>>(
      s.obl, nbl32, s.far_cnt, T, index_bits, node_offsets, far_counts, tree_level_offsets,
      num_levels, level_offsets, s.far_off_node);
  YGX_CHECK_LAUNCH();
  rc = exclusive_scan<int32_t>(s.near_cnt, L, s.near_off, s.scan_tmp, stream);
  if (rc) return rc;
  k_tw_near_tables<<<grid_for(L + 1, 256), 256, 0, stream>>>(s.near_off, s.near_cnt, (int32_t)L,
                                                            index_bits, near_offsets, near_counts);
  YGX_CHECK_LAUNCH();
  if (!ordered) {
    // chunks straight to their rows (offsets taken by the walk), then every
    // row sorted.  Rows sit at their output offsets, or with predicted
    // capacities in their padded slots (in place since the walk) or, when
    // they outgrew them, in an extension behind all slots.
    const int32_t LL = (int32_t)L;
    const int64_t* far_base = s.far_off_node;
    const int64_t* near_base = s.near_off;
    if (pred) {
      for (int pass = 0; pass < 2; ++pass) {
        const bool far = pass == 0;
        const int32_t rows = far ? T : LL;
        const int32_t* cnt = far ? s.far_cnt : s.near_cnt;
        const int32_t* rcap = far ? far_rcap32 : near_rcap32;
        const int64_t* pad = far ? pad_far : pad_near;
        int64_t* roff = far ? s.roff_far : s.roff_near;
        if (rows == 0) continue;
        k_tw_ext_len<<<grid_for(rows, 256), 256, 0, stream>>>(cnt, rcap, rows, s.ext_len);
        YGX_CHECK_LAUNCH();
        rc = exclusive_scan<int32_t>(s.ext_len, rows, s.ext_off, s.scan_tmp, stream);
        if (rc) return rc;
        k_tw_roff<<<grid_for(rows, 256), 256, 0, stream>>>(cnt, rcap, pad, s.ext_off, rows, roff);
        YGX_CHECK_LAUNCH();
        k_tw_prefix_copy<<<kNumSMs * 8, 256, 0, stream>>>(
            cnt, pad, far ? s.first_ovf_far : s.first_ovf_near, s.ext_off, rows,
            far ? far_raw : near_raw, far ? far_raw_cap : near_raw_cap, s.status);
        YGX_CHECK_LAUNCH();
      }
      far_base = s.roff_far;
      near_base = s.roff_near;
    }
    if (far_records > 0) {
      k_tw_copy_raw<<<grid_for((int64_t)far_records * 32, 256, kNumSMs * 16), 256, 0, stream>>>(
          s.far_keys, s.far_recs, (int64_t)far_records, far_base, total, s.far_pool, c.far,
          far_raw, far_raw_cap, s.status);
      YGX_CHECK_LAUNCH();
    }
    if (near_records > 0) {
      k_tw_copy_raw<<<grid_for((int64_t)near_records * 32, 256, kNumSMs * 16), 256, 0, stream>>>(
          s.near_keys, s.near_recs, (int64_t)near_records, near_base, L, s.near_pool, c.near_,
          near_raw, near_raw_cap, s.status);
      YGX_CHECK_LAUNCH();
    }
    const RowTable far_rows{total, s.far_off_node, s.far_cnt, level32, far_raw,
                            pred ? s.roff_far : nullptr, nullptr, sources, targets,
                            target_levels};
    const RowTable near_rows{L, s.near_off, s.near_cnt, nullptr, near_raw,
                             pred ? s.roff_near : nullptr, nullptr, neighbors, nullptr, nullptr};
    rc = row_sort_pass(s.rs, far_rows, near_rows, index_bits, total, stream);
    if (rc) return rc;
  } else {
    // rows: sort the chunk records by (row, class, first id), place them by
    // a scan of their counts, copy
    SortScratch sw;
    {
      Arena sa{(char*)s.sort_ws, 0, s.sort_ws_bytes};
      sw = carve_sort_scratch(sa, c.far_rec > c.near_rec ? c.far_rec : c.near_rec);
    }
    for (int pass = 0; pass < 2; ++pass) {
      const bool far = pass == 0;
      const int64_t m = (int64_t)(far ? far_records : near_records);
      if (m == 0) continue;
      // key bits: row (rank or leaf position) << 32 | class | id
      int64_t rows = far ? total : L;
      int hi_bits = 1;
      while ((1ll << hi_bits) < rows) ++hi_bits;
      rc = onesweep_sort(reinterpret_cast<const uint64_t*>(far ? s.far_keys : s.near_keys),
                         nullptr, m, 0, 32 + hi_bits, reinterpret_cast<uint64_t*>(s.keys_sorted),
                         s.order, sw, false, s.status, stream);
      if (rc) return rc;
      k_tw_sorted_counts<<<grid_for(m, 256), 256, 0, stream>>>(
          s.order, far ? s.far_recs : s.near_recs, m, s.sorted_cnt);
      YGX_CHECK_LAUNCH();
      rc = exclusive_scan<int32_t>(s.sorted_cnt, m, s.dest, s.scan_tmp, stream);
      if (rc) return rc;
      k_tw_copy<<<grid_for(m * 32, 256, kNumSMs * 16), 256, 0, stream>>>(
          s.order, far ? s.far_recs : s.near_recs, m, s.dest, far ? s.far_pool : s.near_pool,
          index_bits, far ? sources : neighbors, far ? targets : nullptr,
          far ? target_levels : nullptr, level32);
      YGX_CHECK_LAUNCH();
    }
  }
  if (max_nbr > 0 && neighbor_leaf_positions && leafpos32 && L > 0) {
    k_tw_nbr_leaf_pos<<<grid_for(L * max_nbr, 256), 256, 0, stream>>>(
        s.near_off, s.near_cnt, L, neighbors, index_bits, leafpos32, max_nbr,
        neighbor_leaf_positions);
    YGX_CHECK_LAUNCH();
  }
  return YGX_OK;
}

// Padded row slots for predicted capacities: pad_far[0..total] and
// pad_near[0..num_leaves] = exclusive sums of far_rcap32 / near_rcap32;
// sums_out (host, 2) = the two totals.  Synchronizes the stream.
size_t ygx_target_pad_workspace_size(int64_t total, int64_t num_leaves) {
  const int64_t m = total > num_leaves ? total : num_leaves;
  return sizeof(int64_t) * ygx::scan_scratch_elems(m > 0 ? m : 1) + 256;
}

int ygx_target_pad(int64_t total, int64_t num_leaves, const int32_t* far_rcap32,
                   const int32_t* near_rcap32, int64_t* pad_far, int64_t* pad_near,
                   uint64_t* sums_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
  using namespace ygx;
  if (total < 1 || num_leaves < 1 || num_leaves > total || !far_rcap32 || !near_rcap32 ||
      !pad_far || !pad_near || !sums_out || !ws ||
      ws_bytes < ygx_target_pad_workspace_size(total, num_leaves))
    return YGX_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(ws) % sizeof(int64_t)) return YGX_ERR_ARG;
  int64_t* tmp = reinterpret_cast<int64_t*>(ws);
  int rc = exclusive_scan<int32_t>(far_rcap32, total, pad_far, tmp, stream);
  if (rc) return rc;
  rc = exclusive_scan<int32_t>(near_rcap32, num_leaves, pad_near, tmp, stream);
  if (rc) return rc;
  int64_t sums[2];
  if (cudaMemcpyAsync(&sums[0], pad_far + total, sizeof(int64_t), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaMemcpyAsync(&sums[1], pad_near + num_leaves, sizeof(int64_t), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  sums_out[0] = (uint64_t)sums[0];
  sums_out[1] = (uint64_t)sums[1];
  return YGX_OK;
}

}  // extern "C"
