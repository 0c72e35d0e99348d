// Symmetric dual-tree traversal (L3): replaces the count walk and the
// compact fill walk of build_interactions_and_neighbors
// (_interactions_impl.py:2600-3558) and the result layouts of
// _result_to_interactions / _result_to_neighbors (:3561-3837).
//
// The pair set is the reference's: a breadth-first refinement of canonical
// (lo, hi) node pairs from (root, root).  Per pair: MAC
// (_interactions_impl.py:338-395) in fp32 in the reference's operation order,
// ACCEPT / NEAR / REFINE (:713-728), split rule on the canonical orientation
// and child pairs (:1262-1310).  An accepted pair lands in both endpoints'
// far rows, a near leaf pair in both leaves' near rows.
//
// Each BFS generation is one launch over the current wavefront.  One walk
// does all the pair work: it counts every far / near row entry (per-node
// counters) and logs
// every accepted or near pair once, as (lo, hi | near-bit), in the CTA's own
// region of a pair log.  A scan of the counts gives the row offsets; a
// scatter pass reads the log back coalesced and writes each pair into both
// endpoints' rows at atomic cursors; the finalize pass sorts every row
// (canonical order) and widens it into the level-major int64/int32 outputs.
#include "rows.cuh"
#include "scan.cuh"

namespace ygx {
namespace {

struct __align__(16) NodeRec {
  float4 c;  // center x, y, z; MAC extent
  int4 k;    // left child, right child (-1 for leaves), leaf position (-1 internal), 0
};

enum MacKind { kMacBH = 0, kMacDehnen = 1, kMacEngblom = 2 };

// stats words (uint64): see ygx.h YGX_TSTAT_*
enum {
  kStatFarTotal = 0,
  kStatNearTotal = 1,
  kStatMaxFar = 2,
  kStatMaxNear = 3,
  kStatAccept = 4,
  kStatNear = 5,
  kStatRefine = 6,
  kStatMaxWf = 7,
  kStatGens = 8,
  kStatWfNeed = 9,
  kStatLogNeed = 10,
  kStatOvfRows = 11,
  kStatOvfEntries = 12,
  kStatExtFar = 13,
  kStatExtNear = 14,
  kStatWords = 16
};

__global__ void k_node_recs(const float* __restrict__ center, const float* __restrict__ radius,
                            const float* __restrict__ max_extent, const int32_t* __restrict__ left32,
                            const int32_t* __restrict__ right32, const int32_t* __restrict__ leafpos,
                            int64_t total, int mac, float dehnen_scale, NodeRec* __restrict__ recs,
                            uint32_t* __restrict__ status) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    // _build_mac_extents (_interactions_impl.py:993-1061): sphere radius for
    // dehnen/engblom (scaled for dehnen), box max half-extent for bh.  The
    // zero-extent propagation there never fires for positive extents.
    float e = mac == kMacBH ? max_extent[k] : radius[k];
    if (mac == kMacDehnen) e = __fmul_rn(dehnen_scale, e);
    if (!(e > 0.0f)) raise_flag(status, kFlagBadInput);
    NodeRec r;
    r.c = make_float4(center[3 * k], center[3 * k + 1], center[3 * k + 2], e);
    r.k = make_int4(left32[k], right32[k], leafpos[k], 0);
    recs[k] = r;
  }
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Returns a unique absolute position pos[key]++ for every lane with pred,
// one atomic per distinct key in the warp.
__device__ __forceinline__ unsigned long long agg_pos(unsigned long long* pos, int key,
                                                      bool pred) {
  unsigned m = __ballot_sync(0xffffffffu, pred);
  unsigned long long p = 0;
  if (pred) {
    unsigned peers = __match_any_sync(m, key);
    int leader = __ffs(peers) - 1;
    unsigned long long base = 0;
    if (((int)(threadIdx.x & 31)) == leader)
      base = atomicAdd(&pos[key], (unsigned long long)__popc(peers));
    base = __shfl_sync(m, base, leader);
    p = base + __popc(peers & lanemask_lt());
  }
  return p;
}

constexpr int kWalkThreads = 256;
constexpr int kWalkBlocksPerSM = 6;
constexpr int kWalkGrid = kNumSMs * kWalkBlocksPerSM;  // fixed across generations
constexpr int kCoarse = 4096;  // coarse index buckets of a walk generation
static_assert(kWalkGrid < 65536, "coarse index holds region ids as uint16");

// What a walk does with its accepted / near pairs:
//  kWalkLog   count row entries and log each pair once (then k_log_scatter);
//  kWalkCount count row entries only (first walk of the plain two-pass mode);
//  kWalkFill  write both directed entries into the exact rows at atomic
//             cursors (second walk of the plain two-pass mode);
//  kWalkPred  write them into rows of predicted capacity (cursor < row end),
//             logging each directed entry that does not fit as (row key, value)
//             with far rows keyed by node and near rows by total + leaf position.
enum WalkMode { kWalkLog = 0, kWalkCount = 1, kWalkFill = 2, kWalkPred = 3 };

struct RowSink {
  unsigned long long* far_pos;         // cursors (fill / predicted)
  unsigned long long* near_pos;
  const unsigned long long* far_end;   // predicted: row ends
  const unsigned long long* near_end;
  int32_t* far_src;                    // raw rows
  int32_t* near_nbr;
  unsigned long long far_total;        // fill: buffer sizes
  unsigned long long near_total;
};

// One BFS generation.  The wavefront of generation g is split into
// kWalkGrid regions, one per CTA of generation g-1, each holding cnt_in[r]
// pairs at wf_in[r * R ...].  A CTA maps a global input index to (region,
// offset) through the prefix sum of cnt_in kept in shared memory.  Input is
// taken in 32-pair warp chunks interleaved across CTAs (chunk c goes to CTA
// c mod G), and a CTA appends child pairs to its own wavefront region and
// accepted / near pairs to its own log region (which grows over all
// generations, log_cnt[b] entries so far) in a fixed order (iteration,
// warp, lane) with one barrier per iteration.  The walk is therefore
// deterministic, and the entries a region would have needed are counted
// even past its end, so one re-run with the reported sizes always fits.
template <int kMode, int kMac>
__global__ void __launch_bounds__(kWalkThreads, kWalkBlocksPerSM)
    k_walk_gen(const NodeRec* __restrict__ nodes, int32_t ni, int32_t total_nodes,
               float theta_sq, float theta,
               const int2* __restrict__ wf_in, int2* __restrict__ wf_out,
               const uint32_t* __restrict__ cnt_in, uint32_t* __restrict__ cnt_out, uint32_t R,
               uint32_t* __restrict__ sizes, int gen, int32_t* __restrict__ far_cnt,
               int32_t* __restrict__ near_cnt, int2* __restrict__ log,
               unsigned long long* __restrict__ log_cnt, unsigned long long LR, RowSink sink,
               unsigned long long* __restrict__ stats, uint32_t* __restrict__ status) {
  constexpr int kWarps = kWalkThreads / 32;
  __shared__ uint32_t s_prefix[kWalkGrid + 1];
  __shared__ uint16_t s_coarse[kCoarse];
  __shared__ uint32_t s_wsum[kWarps];
  __shared__ uint32_t s_wt[2][kWarps];
  const int G = gridDim.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // Exclusive prefix of the input region counts (G <= kWalkGrid).
  {
    constexpr int kPer = (kWalkGrid + kWalkThreads - 1) / kWalkThreads;
    uint32_t v[kPer];
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int r = tid * kPer + k;
      v[k] = r < G ? cnt_in[r] : 0u;
      mine += v[k];
    }
    uint32_t incl = mine;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += o;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += s_wsum[w];
    uint32_t run = wpre + incl - mine;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int r = tid * kPer + k;
      if (r < G) s_prefix[r] = run;
      run += v[k];
    }
    if (tid == kWalkThreads - 1) s_prefix[G] = run;
    __syncthreads();
  }
  const uint32_t total_in = s_prefix[G];
  if (total_in == 0) {
    if (tid == 0) cnt_out[blockIdx.x] = 0;
    return;
  }
  // Coarse index: s_coarse[j] = region holding index j << shift (buckets of
  // 2^shift indices, at most kCoarse of them), so a lookup starts at most a
  // bucket's worth of regions before its target.
  int shift = 0;
  while (((total_in - 1) >> shift) >= (uint32_t)kCoarse) ++shift;
  for (int r = tid; r < G; r += kWalkThreads) {
    const uint32_t mask = (1u << shift) - 1;
    const uint32_t j0 = (uint32_t)(((uint64_t)s_prefix[r] + mask) >> shift);
    const uint32_t j1 = (uint32_t)(((uint64_t)s_prefix[r + 1] + mask) >> shift);
    for (uint32_t j = j0; j < j1; ++j) s_coarse[j] = (uint16_t)r;
  }
  __syncthreads();
  int2* my_out = wf_out + (size_t)blockIdx.x * R;
  unsigned long long n_acc = 0, n_near = 0, n_ref = 0;
  unsigned long long cta_base = 0;  // block-uniform: pairs appended so far
  unsigned long long log_base = log_cnt[blockIdx.x];  // block-uniform
  const uint32_t nchunks = (total_in + 31) >> 5;
  const uint32_t cstride = (uint32_t)kWarps * G;
  int buf = 0;
  for (uint32_t chunk0 = blockIdx.x; chunk0 < nchunks; chunk0 += cstride, buf ^= 1) {
    // chunk0 is warp 0's chunk (block-uniform loop); this warp takes chunk
    const uint32_t chunk = chunk0 + warp * G;
    const bool wvalid = chunk < nchunks;
    const uint32_t wbase = chunk << 5;
    const uint32_t i = wbase + lane;
    const bool valid = wvalid && i < total_in;
    int t = 0, sv = 0;
    if (valid) {
      // Region of i: from the coarse index of the warp's first index, step
      // past the regions that end at or before i.
      int r = s_coarse[wbase >> shift];
      while (r + 1 < G && s_prefix[r + 1] <= i) ++r;
      const int2 p = wf_in[(size_t)r * R + (i - s_prefix[r])];
      t = p.x;
      sv = p.y;
    }
    const bool in_range = (unsigned)t < (unsigned)total_nodes &&
                          (unsigned)sv < (unsigned)total_nodes;
    if (valid && !in_range) raise_flag(status, kFlagBadInput);
    const bool live = valid && in_range;
    NodeRec A, B;
    if (live) {
      A = nodes[t];
      B = nodes[sv];
    } else {
      A.c = make_float4(0.f, 0.f, 0.f, 0.f);
      A.k = make_int4(-1, -1, 0, 0);
      B = A;
    }
    bool acc = false, nearp = false, refine = false;
    if (live) {
      const float dx = __fsub_rn(A.c.x, B.c.x);
      const float dy = __fsub_rn(A.c.y, B.c.y);
      const float dz = __fsub_rn(A.c.z, B.c.z);
      float d2 = __fmul_rn(dx, dx);
      d2 = __fadd_rn(d2, __fmul_rn(dy, dy));
      d2 = __fadd_rn(d2, __fmul_rn(dz, dz));
      const float et = A.c.w, es = B.c.w;
      bool ok;
      if (kMac == kMacEngblom) {
        const float big = fmax_nan(et, es), small = fmin_nan(et, es);
        const float lhs = __fadd_rn(big, __fmul_rn(theta, small));
        ok = __fmul_rn(lhs, lhs) <= __fmul_rn(theta_sq, d2);
      } else {
        const float sum = __fadd_rn(et, es);
        ok = __fmul_rn(sum, sum) <= __fmul_rn(theta_sq, d2);
      }
      const bool diff = t != sv;
      acc = diff && d2 > 0.0f && ok;
      // leaves carry -1 children (node records), in a single tree and a forest
      nearp = !acc && diff && A.k.x < 0 && B.k.x < 0;
      refine = !acc && !nearp;
    }
    n_acc += acc;
    n_near += nearp;
    n_ref += refine;
    int lc = 0;  // log entries of this lane
    int2 le0 = make_int2(0, 0), le1 = le0;
    if (kMode == kWalkLog || kMode == kWalkCount) {
      // Row counts: plain fire-and-forget atomics (aggregating equal keys in
      // the warp with match-any first measured slower here).
      if (acc) {
        atomicAdd(&far_cnt[t], 1);
        atomicAdd(&far_cnt[sv], 1);
      }
      if (nearp) {
        atomicAdd(&near_cnt[A.k.z], 1);
        atomicAdd(&near_cnt[B.k.z], 1);
      }
      if (kMode == kWalkLog && (acc || nearp)) {
        lc = 1;
        le0 = make_int2(t, sv | (nearp ? (int)0x80000000u : 0));
      }
    } else if (acc || nearp) {
      const int rt = acc ? t : A.k.z, rs = acc ? sv : B.k.z;
      unsigned long long* cur = acc ? sink.far_pos : sink.near_pos;
      int32_t* dst = acc ? sink.far_src : sink.near_nbr;
      const unsigned long long pt = atomicAdd(&cur[rt], 1ull);
      const unsigned long long ps = atomicAdd(&cur[rs], 1ull);
      if (kMode == kWalkFill) {
        const unsigned long long lim = acc ? sink.far_total : sink.near_total;
        const uint32_t fl = acc ? kFlagFarOverflow : kFlagNearOverflow;
        if (pt < lim) dst[pt] = sv; else raise_flag(status, fl);
        if (ps < lim) dst[ps] = t; else raise_flag(status, fl);
      } else {
        const unsigned long long* end = acc ? sink.far_end : sink.near_end;
        const int kt = acc ? t : total_nodes + rt, ks = acc ? sv : total_nodes + rs;
        if (pt < end[rt]) {
          dst[pt] = sv;
        } else {
          le0 = make_int2(kt, sv);
          lc = 1;
        }
        if (ps < end[rs]) {
          dst[ps] = t;
        } else if (lc == 0) {
          le0 = make_int2(ks, t);
          lc = 1;
        } else {
          le1 = make_int2(ks, t);
          lc = 2;
        }
      }
    }

    // Children of a refined pair (_interactions_impl.py:1262-1310).
    int nc = 0;
    int2 c0 = make_int2(0, 0), c1 = c0, c2 = c0, c3 = c0;
    if (refine) {
      const bool same = t == sv;
      const bool t_int = A.k.x >= 0, s_int = B.k.x >= 0;
      const float et = A.c.w, es = B.c.w;
      const bool split_t = t_int && (same || !s_int || et >= es);
      const bool split_s = s_int && (same || !t_int || es > et);
      auto mk = [](int a, int b) { return a < b ? make_int2(a, b) : make_int2(b, a); };
      if (split_t && split_s) {
        if (same) {
          c0 = mk(A.k.x, A.k.x);
          c1 = mk(A.k.x, A.k.y);
          c2 = mk(A.k.y, A.k.y);
          nc = 3;
        } else {
          c0 = mk(A.k.x, B.k.x);
          c1 = mk(A.k.x, B.k.y);
          c2 = mk(A.k.y, B.k.x);
          c3 = mk(A.k.y, B.k.y);
          nc = 4;
        }
      } else if (split_t) {
        c0 = mk(A.k.x, sv);
        c1 = mk(A.k.y, sv);
        nc = 2;
      } else if (split_s) {
        c0 = mk(t, B.k.x);
        c1 = mk(t, B.k.y);
        nc = 2;
      }
    }
    // warp scan of (children | log entries << 8): <= 128 and <= 64 per warp
    int incl = nc | (lc << 8);
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      int v = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += v;
    }
    // children (<= 1024 per CTA) in the low half, log entries in the high
    if (lane == 31)
      s_wt[buf][warp] = (uint32_t)(incl & 0xff) | ((uint32_t)(incl >> 8) << 16);
    __syncthreads();
    uint32_t pre = 0, sum = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t v = s_wt[buf][w];
      pre += w < warp ? v : 0u;
      sum += v;
    }
    if (lc > 0) {
      const unsigned long long la = log_base + (pre >> 16) + (uint32_t)((incl >> 8) - lc);
      int2* lp = log + (size_t)blockIdx.x * LR;
      if (la < LR) lp[la] = le0; else raise_flag(status, kFlagLogOverflow);
      if (lc > 1) {
        if (la + 1 < LR) lp[la + 1] = le1; else raise_flag(status, kFlagLogOverflow);
      }
    }
    log_base += sum >> 16;
    sum &= 0xffffu;
    pre &= 0xffffu;
    // Every child that fits is written, so the first min(total, R) slots of
    // the region are always filled.
    const unsigned long long at = cta_base + pre + (uint32_t)((incl & 0xff) - nc);
    if (nc > 0) {
      if (at + (unsigned long long)nc <= R) {
        int2* o = my_out + at;
        o[0] = c0;
        if (nc > 1) o[1] = c1;
        if (nc > 2) o[2] = c2;
        if (nc > 3) o[3] = c3;
      } else {
        if (at + 0 < R) my_out[at + 0] = c0;
        if (nc > 1 && at + 1 < R) my_out[at + 1] = c1;
        if (nc > 2 && at + 2 < R) my_out[at + 2] = c2;
        raise_flag(status, kFlagQueueOverflow);
      }
    }
    cta_base += sum;
  }
  if (tid == 0) {
    const uint32_t c = cta_base < R ? (uint32_t)cta_base : R;
    cnt_out[blockIdx.x] = c;
    if (c) atomicAdd(&sizes[gen + 1], c);
    log_cnt[blockIdx.x] = log_base;
    atomicMax(&stats[kStatWfNeed], cta_base);
  }
  for (int o = 16; o > 0; o >>= 1) {
    n_acc += __shfl_xor_sync(0xffffffffu, n_acc, o);
    n_near += __shfl_xor_sync(0xffffffffu, n_near, o);
    n_ref += __shfl_xor_sync(0xffffffffu, n_ref, o);
  }
  if (lane == 0) {
    if (n_acc) atomicAdd(&stats[kStatAccept], n_acc);
    if (n_near) atomicAdd(&stats[kStatNear], n_near);
    if (n_ref) atomicAdd(&stats[kStatRefine], n_ref);
  }
}

__global__ void k_init_cursors(const int64_t* __restrict__ far_off, int64_t total,
                               unsigned long long* __restrict__ far_pos,
                               const int64_t* __restrict__ near_off, int64_t L,
                               unsigned long long* __restrict__ near_pos) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    far_pos[k] = (unsigned long long)far_off[k];
    if (k < L) near_pos[k] = (unsigned long long)near_off[k];
  }
}

// Scatter pass: CTA b reads its log region back in order and writes each
// pair into both endpoints' rows.  Far rows (keys 0..total-1) and near rows
// (keys total + leaf position) share one cursor array, so every entry makes
// two warp-aggregated cursor claims whatever its kind.  Cursors start at each
// row's offset, so the claim yields the write position; k_check_cursors then
// verifies every row ended exactly at its end.  Nothing past the totals is
// written.
__global__ void __launch_bounds__(256)
    k_log_scatter(const int2* __restrict__ log, const unsigned long long* __restrict__ log_cnt,
                  unsigned long long LR, const int32_t* __restrict__ leafpos, int32_t total,
                  unsigned long long* __restrict__ pos, unsigned long long far_total,
                  unsigned long long near_total, int32_t* __restrict__ far_src,
                  int32_t* __restrict__ near_nbr, uint32_t* __restrict__ status,
                  uint32_t skip_mask) {
  if (*status & skip_mask) return;  // flagged before the scatter: write nothing
  const int lane = threadIdx.x & 31;
  for (int b = blockIdx.x; b < kWalkGrid; b += gridDim.x) {
    const unsigned long long n = log_cnt[b] < LR ? log_cnt[b] : LR;
    const int2* src = log + (size_t)b * LR;
    for (unsigned long long base = threadIdx.x & ~31u; base < n; base += blockDim.x) {
      const unsigned long long i = base + lane;
      int t = 0, sv = 0;
      bool act = false, nearp = false;
      if (i < n) {
        const int2 e = src[i];
        t = e.x;
        sv = e.y & 0x7fffffff;
        nearp = e.y < 0;
        act = true;
      }
      const int kt = act ? (nearp ? total + leafpos[t] : t) : 0;
      const int ks = act ? (nearp ? total + leafpos[sv] : sv) : 0;
      const unsigned long long pt = agg_pos(pos, kt, act);
      const unsigned long long ps = agg_pos(pos, ks, act);
      if (act) {
        int32_t* dst = nearp ? near_nbr : far_src;
        const unsigned long long lim = nearp ? near_total : far_total;
        const uint32_t fl = nearp ? kFlagNearOverflow : kFlagFarOverflow;
        if (pt < lim) dst[pt] = sv; else raise_flag(status, fl);
        if (ps < lim) dst[ps] = t; else raise_flag(status, fl);
      }
    }
  }
}

// ---- predicted mode ----------------------------------------------------------

__global__ void k_pad_ends(const int64_t* __restrict__ pad, const int32_t* __restrict__ cap,
                           int64_t n, unsigned long long* __restrict__ end,
                           unsigned long long* __restrict__ pos) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    end[k] = (unsigned long long)(pad[k] + cap[k]);
    pos[k] = (unsigned long long)pad[k];
  }
}

// Exact row lengths from the cursors of the predicted walk; rows that
// outgrew their capacity get their full length in ext_cnt (they move to the
// extension area), the others 0.
__global__ void k_pred_counts(const unsigned long long* __restrict__ pos,
                              const int64_t* __restrict__ pad, const int32_t* __restrict__ cap,
                              int64_t n, int32_t* __restrict__ cnt, int32_t* __restrict__ ext_cnt,
                              unsigned long long* __restrict__ stats, int ext_word) {
  unsigned long long rows = 0, entries = 0, ext = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = (int64_t)pos[k] - pad[k];
    cnt[k] = (int32_t)c;
    const bool over = c > cap[k];
    ext_cnt[k] = over ? (int32_t)c : 0;
    if (over) {
      ++rows;
      entries += (unsigned long long)(c - cap[k]);
      ext += (unsigned long long)c;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    rows += __shfl_xor_sync(0xffffffffu, rows, o);
    entries += __shfl_xor_sync(0xffffffffu, entries, o);
    ext += __shfl_xor_sync(0xffffffffu, ext, o);
  }
  if ((threadIdx.x & 31) == 0 && rows) {
    atomicAdd(&stats[kStatOvfRows], rows);
    atomicAdd(&stats[kStatOvfEntries], entries);
    atomicAdd(&stats[ext_word], ext);
  }
}

// Read offsets of the raw rows: the padded row, or for a row that outgrew
// its capacity a fresh place in the extension area (after all padded rows)
// that will hold its first cap entries (k_relocate_copy) followed by the
// entries the walk logged (appended at the cursor left at ext + cap).  Rows
// that move are listed for the copy.
__global__ void k_relocate_mark(const int64_t* __restrict__ pad, const int32_t* __restrict__ cap,
                                const int32_t* __restrict__ ext_cnt,
                                const int64_t* __restrict__ ext_off, int64_t n, int64_t raw_cap,
                                unsigned long long* __restrict__ pos,
                                int64_t* __restrict__ raw_off, int32_t* __restrict__ moved,
                                uint32_t* __restrict__ n_moved, uint32_t* __restrict__ status,
                                uint32_t overflow_flag) {
  const int64_t ext_base = pad[n];
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (ext_cnt[k] == 0) {
      raw_off[k] = pad[k];
      continue;
    }
    const int64_t dst = ext_base + ext_off[k];
    if (dst + ext_cnt[k] > raw_cap) {
      raise_flag(status, overflow_flag);
      raw_off[k] = pad[k];
      continue;
    }
    raw_off[k] = dst;
    pos[k] = (unsigned long long)(dst + cap[k]);
    moved[atomicAdd(n_moved, 1u)] = (int32_t)k;
  }
}

// One CTA per moved row copies its first cap entries to the extension area.
__global__ void __launch_bounds__(256)
    k_relocate_copy(const int32_t* __restrict__ moved, const uint32_t* __restrict__ n_moved,
                    const int64_t* __restrict__ pad, const int32_t* __restrict__ cap,
                    const int64_t* __restrict__ raw_off, int32_t* __restrict__ raw) {
  const uint32_t nm = *n_moved;
  for (uint32_t b = blockIdx.x; b < nm; b += gridDim.x) {
    const int32_t k = moved[b];
    const int64_t src = pad[k], dst = raw_off[k];
    for (int64_t e = threadIdx.x; e < cap[k]; e += blockDim.x) raw[dst + e] = raw[src + e];
  }
}

// Logged overflow entries (row key, value) -> their rows' extension tails.
__global__ void k_ovf_scatter(const int2* __restrict__ log,
                              const unsigned long long* __restrict__ log_cnt,
                              unsigned long long LR, int32_t total,
                              unsigned long long* __restrict__ far_pos,
                              unsigned long long* __restrict__ near_pos,
                              int32_t* __restrict__ far_raw, int32_t* __restrict__ near_raw,
                              const int64_t* __restrict__ far_end,
                              const int64_t* __restrict__ near_end,
                              uint32_t* __restrict__ status) {
  for (int b = blockIdx.x; b < kWalkGrid; b += gridDim.x) {
    const unsigned long long n = log_cnt[b] < LR ? log_cnt[b] : LR;
    const int2* src = log + (size_t)b * LR;
    for (unsigned long long i = threadIdx.x; i < n; i += blockDim.x) {
      const int2 e = src[i];
      if (e.x < total) {
        const unsigned long long p = atomicAdd(&far_pos[e.x], 1ull);
        if ((long long)p < far_end[e.x]) far_raw[p] = e.y;
        else raise_flag(status, kFlagFarOverflow);
      } else {
        const int r = e.x - total;
        const unsigned long long p = atomicAdd(&near_pos[r], 1ull);
        if ((long long)p < near_end[r]) near_raw[p] = e.y;
        else raise_flag(status, kFlagNearOverflow);
      }
    }
  }
}

// Row end for the extension tails: raw_off + count.
__global__ void k_raw_ends(const int64_t* __restrict__ raw_off, const int32_t* __restrict__ cnt,
                           int64_t n, int64_t* __restrict__ end) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    end[k] = raw_off[k] + cnt[k];
}

// Every relocated row's cursor must end at its row end.
__global__ void k_check_ext(const unsigned long long* __restrict__ pos,
                            const int64_t* __restrict__ end, const int32_t* __restrict__ ext_cnt,
                            int64_t n, uint32_t* __restrict__ status, uint32_t flag) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    if (ext_cnt[k] && (long long)pos[k] != end[k]) raise_flag(status, flag);
}

// Every cursor must end exactly at its row's end (fill == count).
__global__ void k_check_cursors(const int64_t* __restrict__ far_off,
                                const int32_t* __restrict__ far_cnt,
                                const unsigned long long* __restrict__ far_pos, int64_t total,
                                const int64_t* __restrict__ near_off,
                                const int32_t* __restrict__ near_cnt,
                                const unsigned long long* __restrict__ near_pos, int64_t L,
                                uint32_t* __restrict__ status) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (far_pos[k] != (unsigned long long)(far_off[k] + far_cnt[k]))
      raise_flag(status, kFlagFarOverflow);
    if (k < L && near_pos[k] != (unsigned long long)(near_off[k] + near_cnt[k]))
      raise_flag(status, kFlagNearOverflow);
  }
}

__global__ void k_seed(int2* wf, uint32_t* cnt, uint32_t* sizes, int root) {
  // generation 0: one pair (root, root) in region 0, all other regions empty
  for (int r = threadIdx.x; r < kWalkGrid; r += blockDim.x) cnt[r] = r == 0 ? 1u : 0u;
  if (threadIdx.x == 0) {
    wf[0] = make_int2(root, root);
    sizes[0] = 1;
  }
}

// Generation 0 of a forest walk: (root_s, root_s) for every set, spread
// over the regions round-robin.  root_s = 2 leaf_off[s] - s, or for a set
// flagged malformed its first node without a parent (the reference starts
// its walk at argmin(parent)).
__global__ void k_seed_forest(int2* wf, uint32_t* cnt, uint32_t* sizes, uint32_t R, int G,
                              const int64_t* __restrict__ leaf_off, int64_t S,
                              const int32_t* __restrict__ parent32,
                              const uint32_t* __restrict__ seg_flags,
                              uint32_t* __restrict__ status) {
  // regions 0 .. G-1 (G = the walk's grid) hold the seeds, the rest stay empty
  for (int r = threadIdx.x; r < kWalkGrid; r += blockDim.x) {
    const int64_t c = r < G && S > r ? (S - r + G - 1) / G : 0;
    cnt[r] = c <= R ? (uint32_t)c : R;
    if (c > R) raise_flag(status, kFlagQueueOverflow);
  }
  for (int64_t sg = threadIdx.x; sg < S; sg += blockDim.x) {
    const int64_t a = leaf_off[sg], Ls = leaf_off[sg + 1] - a, NO = 2 * a - sg;
    int64_t root = NO;
    if (seg_flags && (seg_flags[sg] & kFlagMalformed)) {
      for (int64_t k = NO; k < NO + 2 * Ls - 1; ++k)
        if (parent32[k] < 0) { root = k; break; }
    }
    const int64_t r = sg % G, k = sg / G;
    if (k < R) wf[(size_t)r * R + k] = make_int2((int)root, (int)root);
  }
  if (threadIdx.x == 0) sizes[0] = (uint32_t)S;
}

// Totals and maxima of the count pass; max wavefront and generations.
__global__ void k_count_stats(const int32_t* __restrict__ far_cnt, int64_t total,
                              const int32_t* __restrict__ near_cnt, int64_t L,
                              const uint32_t* __restrict__ sizes, int max_gens,
                              const unsigned long long* __restrict__ log_cnt,
                              unsigned long long* __restrict__ stats) {
  unsigned long long fsum = 0, nsum = 0, fmax = 0, nmax = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long v = (unsigned long long)far_cnt[k];
    fsum += v;
    fmax = v > fmax ? v : fmax;
  }
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < L;
       k += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long v = (unsigned long long)near_cnt[k];
    nsum += v;
    nmax = v > nmax ? v : nmax;
  }
  for (int off = 16; off > 0; off >>= 1) {
    fsum += __shfl_xor_sync(0xffffffffu, fsum, off);
    nsum += __shfl_xor_sync(0xffffffffu, nsum, off);
    unsigned long long a = __shfl_xor_sync(0xffffffffu, fmax, off);
    unsigned long long b = __shfl_xor_sync(0xffffffffu, nmax, off);
    fmax = a > fmax ? a : fmax;
    nmax = b > nmax ? b : nmax;
  }
  if ((threadIdx.x & 31) == 0) {
    if (fsum) atomicAdd(&stats[kStatFarTotal], fsum);
    if (nsum) atomicAdd(&stats[kStatNearTotal], nsum);
    atomicMax(&stats[kStatMaxFar], fmax);
    atomicMax(&stats[kStatMaxNear], nmax);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long mw = 1, g = 0;
    for (int k = 0; k <= max_gens; ++k) {
      if (sizes[k] == 0) break;
      g = k + 1;
      if (k > 0 && sizes[k] > mw) mw = sizes[k];
    }
    stats[kStatMaxWf] = mw;
    stats[kStatGens] = g;
    // capacities (in total entries over all regions) that would have fit
    unsigned long long ln = 0;
    for (int b = 0; b < kWalkGrid; ++b) ln = log_cnt[b] > ln ? log_cnt[b] : ln;
    stats[kStatLogNeed] = ln * kWalkGrid;
    stats[kStatWfNeed] = stats[kStatWfNeed] * kWalkGrid;
  }
}

// counts in nodes_by_level order (for the level-major far layout).
__global__ void k_gather_counts(const int32_t* __restrict__ cnt, const int32_t* __restrict__ order,
                                int64_t m, int32_t* __restrict__ out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x)
    out[r] = cnt[order ? order[r] : r];
}

// node_offsets[nbl[r]] = obl[r]; far_off (int64, node-indexed) the same;
// counts widened; level_offsets = obl[tree_level_offsets[l]].
// After a walk of a fixed number of generations (no host probe): flags what
// the caller's fixed sizes cannot hold -- a wavefront still non-empty after
// the last generation, directed totals above the output capacities -- and
// k_zero_counts_if then zeroes every row count, so the offset, scatter and
// finalize stages that follow write nothing.
__global__ void k_guard_totals(const uint32_t* __restrict__ sizes, int gens,
                               const unsigned long long* __restrict__ stats,
                               unsigned long long far_cap, unsigned long long near_cap,
                               uint32_t* __restrict__ status) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (sizes[gens] != 0) raise_flag(status, kFlagQueueOverflow);
  if (stats[kStatFarTotal] > far_cap) raise_flag(status, kFlagFarOverflow);
  if (stats[kStatNearTotal] > near_cap) raise_flag(status, kFlagNearOverflow);
}

__global__ void k_zero_counts_if(const uint32_t* __restrict__ status, uint32_t mask,
                                 int32_t* __restrict__ far_cnt, int64_t total,
                                 int32_t* __restrict__ near_cnt, int64_t L) {
  if ((*status & mask) == 0) return;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    far_cnt[k] = 0;
    if (k < L) near_cnt[k] = 0;
  }
}

__global__ void k_far_offsets(const int64_t* __restrict__ obl, const int32_t* __restrict__ nbl,
                              const int32_t* __restrict__ cnt, int64_t total, int index_bits,
                              int64_t* __restrict__ far_off, void* node_offsets, void* counts_out,
                              const void* tree_level_offsets, int num_levels,
                              void* level_offsets_out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= total;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (r == total) {
      store_idx(node_offsets, index_bits, total, obl[total]);
    } else {
      const int32_t v = nbl[r];
      far_off[v] = obl[r];
      store_idx(node_offsets, index_bits, v, obl[r]);
      store_idx(counts_out, index_bits, r, cnt[r]);
    }
    if (r <= num_levels) {
      int64_t li = load_idx(tree_level_offsets, index_bits, r);
      store_idx(level_offsets_out, index_bits, r, obl[li]);
    }
  }
}

__global__ void k_near_offsets(const int64_t* __restrict__ off, const int32_t* __restrict__ cnt,
                               int64_t L, int index_bits, void* offsets_out, void* counts_out) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j <= L;
       j += (int64_t)gridDim.x * blockDim.x) {
    store_idx(offsets_out, index_bits, j, off[j]);
    if (j < L) store_idx(counts_out, index_bits, j, cnt[j]);
  }
}

// ---------------------------------------------------------------------------
// Row finalize: sort each row ascending and widen it.  The network is the
// all-ascending ("mirrored") bitonic sort: for each block size k the first
// step pairs i with i ^ (k - 1), later steps pair i with i ^ j.  Every
// comparator puts the minimum at the lower index, so a row of any length n
// sorts as if padded with +inf, and comparators whose upper index is >= n
// are no-ops that can be skipped -- no padding storage is needed.
// Rows up to kWarpRowCap entries: one warp in shared memory; up to
// kBlockRowCap: one CTA in shared memory; longer: one CTA in place in
// global memory.

constexpr int kWarpRowCap = 1024;   // one warp, 4 KB of shared memory
constexpr int kBlockRowCap = 16384; // one CTA, 64 KB of shared memory
constexpr int kBigThreads = 512;

template <bool kBlockSync>
__device__ __forceinline__ void mirrored_bitonic(int32_t* a, int64_t n64, int tid, int nthreads) {
  // Row lengths stay below 2^31 (they are counts of one node's partners).
  const int32_t n = (int32_t)n64;
  int32_t np2 = 1;
  while (np2 < n) np2 <<= 1;
  for (int32_t k = 2; k <= np2; k <<= 1) {
    for (int32_t j = k >> 1; j > 0; j >>= 1) {
      const bool first = j == (k >> 1);
      // np2 / 2 comparators per step; comparator c -> lower index i
      for (int32_t c = tid; c < (np2 >> 1); c += nthreads) {
        // j is a power of two: insert a zero bit at position log2(j).
        const int32_t i = ((c & ~(j - 1)) << 1) | (c & (j - 1));
        const int32_t p = first ? (i ^ (k - 1)) : (i | j);
        const int32_t lo = i < p ? i : p, hi = i < p ? p : i;
        if (hi < n) {
          const int32_t x = a[lo], y = a[hi];
          if (x > y) { a[lo] = y; a[hi] = x; }
        }
      }
      if (kBlockSync) __syncthreads(); else __syncwarp();
    }
  }
}

// Writes the sorted row: values (sources or neighbours) in the index dtype
// and, for far rows, the target node and its level for every entry.
__device__ __forceinline__ void emit_row(const int32_t* a, int64_t n, int64_t off, int index_bits,
                                         void* vals_out, void* tgt_out, void* lvl_out, int32_t tgt,
                                         int32_t vbase,
                                         int32_t lvl, int tid, int nthreads) {
  for (int64_t k = tid; k < n; k += nthreads) {
    store_idx(vals_out, index_bits, off + k, a[k] - vbase);
    if (tgt_out) {
      store_idx(tgt_out, index_bits, off + k, tgt);
      store_idx(lvl_out, index_bits, off + k, lvl);
    }
  }
}

// One warp sorts a row of up to 32*R entries held in registers in the
// "blocked" layout: lane l holds elements l*R .. l*R+R-1.  Loads and stores
// stay coalesced through a padded shared-memory transpose (row stride R+1,
// conflict-free both ways).  With this layout the bitonic steps with
// partner distance j < R are compare-exchanges between registers of one
// lane and only the steps with j >= R exchange across lanes (shuffles).
// The row is padded with INT32_MAX to 32*R entries.
template <int R>
__device__ __forceinline__ void warp_sort_row(const int32_t* __restrict__ raw, int64_t roff,
                                              int64_t off,
                                              int n, int index_bits, void* vals_out,
                                              void* tgt_out, void* lvl_out, int32_t tgt,
                                              int32_t vbase, int32_t lvl, int lane,
                                              int32_t* __restrict__ sm) {
  constexpr int S = R + 1;
  constexpr int LOGR = R == 1 ? 0 : R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : R == 16 ? 4 : 5;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int e = r * 32 + lane;
    sm[(e >> LOGR) * S + (e & (R - 1))] = e < n ? raw[roff + e] : INT32_MAX;
  }
  __syncwarp();
  int32_t v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = sm[lane * S + r];
  // All-ascending network: every comparator puts the minimum at the lower
  // index, so no per-comparator direction is needed.  The first step of a
  // k-block pairs i with i ^ (k - 1): inside a lane register r with r ^
  // (k - 1) while k <= R, else lane l ^ (k / R - 1), register R - 1 - r.
#pragma unroll
  for (int k = 2; k <= 32 * R; k <<= 1) {
    if (k <= R) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int rp = r ^ (k - 1);
        if (rp > r) {
          const int32_t x = v[r], y = v[rp];
          v[r] = min(x, y);
          v[rp] = max(x, y);
        }
      }
    } else {
      const int m = (k >> LOGR) - 1;
      const bool lower = (lane & ((k >> LOGR) >> 1)) == 0;
      int32_t y[R];
#pragma unroll
      for (int r = 0; r < R; ++r) y[r] = __shfl_xor_sync(0xffffffffu, v[R - 1 - r], m);
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = lower ? min(v[r], y[r]) : max(v[r], y[r]);
    }
#pragma unroll
    for (int j = k >> 2; j > 0; j >>= 1) {
      if (j < R) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if ((r & j) == 0) {
            const int rp = r | j;
            const int32_t x = v[r], y = v[rp];
            v[r] = min(x, y);
            v[rp] = max(x, y);
          }
        }
      } else {
        const int lj = j >> LOGR;
        const bool lower = (lane & lj) == 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int32_t y = __shfl_xor_sync(0xffffffffu, v[r], lj);
          v[r] = lower ? min(v[r], y) : max(v[r], y);
        }
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int r = 0; r < R; ++r) sm[lane * S + r] = v[r];
  __syncwarp();
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int e = r * 32 + lane;
    if (e < n) {
      const int32_t x = sm[(e >> LOGR) * S + (e & (R - 1))];
      store_idx(vals_out, index_bits, off + e, x - vbase);
      if (tgt_out) {
        store_idx(tgt_out, index_bits, off + e, tgt);
        store_idx(lvl_out, index_bits, off + e, lvl);
      }
    }
  }
  __syncwarp();
}

// Rows are bucketed by size class first; each class runs in its own kernel
// with a single register-network instantiation (one instantiation per
// kernel keeps the instruction footprint small).  Class c holds rows of
// 32*2^(c-1) < n <= 32*2^c entries (c = 0: n <= 32); longer rows go to the
// CTA kernel.
constexpr int kRowClasses = 6;  // R = 1, 2, 4, 8, 16, 32

// Rows of two tables in one pass: row r < ta.rows is ta's row r, the others
// are tb's row r - ta.rows.
__global__ void k_rows_classify(RowTable ta, RowTable tb, int32_t* __restrict__ lists,
                                int64_t list_stride, uint32_t* __restrict__ list_n,
                                int32_t* __restrict__ big_rows, uint32_t* __restrict__ n_big) {
  const int64_t rows = ta.rows + tb.rows;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int n = r < ta.rows ? ta.cnt[r] : tb.cnt[r - ta.rows];
    if (n == 0) continue;
    if (n > kWarpRowCap) {
      // rows longer than kBlockRowCap from the front, the others from the
      // back: the long-row kernel takes the longest first
      if (n > kBlockRowCap) big_rows[atomicAdd(&n_big[0], 1u)] = (int32_t)r;
      else big_rows[list_stride - 1 - atomicAdd(&n_big[8], 1u)] = (int32_t)r;
      continue;
    }
    int c = 0;
    while ((32 << c) < n) ++c;
    // warp-aggregated append per class
    const unsigned m = __activemask();
    const unsigned peers = __match_any_sync(m, c);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&list_n[c], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    lists[c * list_stride + base + __popc(peers & lt)] = (int32_t)r;
  }
}

template <int R>
__global__ void __launch_bounds__(256, R >= 32 ? 2 : (R >= 16 ? 3 : 4))
    k_rows_class(const int32_t* __restrict__ list, const uint32_t* __restrict__ list_n,
                 RowTable ta, RowTable tb, int index_bits) {
  __shared__ int32_t s_rows[8][32 * (R + 1)];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t nm = *list_n;
  for (uint32_t b = blockIdx.x * 8 + w; b < nm; b += gridDim.x * 8) {
    const int32_t g = list[b];
    const bool second = g >= ta.rows;
    const RowTable& T = second ? tb : ta;
    const int32_t r = second ? g - (int32_t)ta.rows : g;
    const int32_t vbase = T.rbase ? T.rbase[r] : 0;
    warp_sort_row<R>(T.raw, T.roff ? T.roff[r] : T.off[r], T.off[r], T.cnt[r], index_bits,
                     T.vals, T.tgts, T.lvls, r - vbase, vbase, T.lvl ? T.lvl[r] : 0, lane,
                     s_rows[w]);
  }
}

// Position of the r-th (0-based) set bit of w (r < popc(w)), by halving.
__device__ __forceinline__ int select_bit(uint32_t w, int r) {
  int base = 0;
  int c = __popc(w & 0xffffu);
  if (r >= c) { r -= c; w >>= 16; base += 16; }
  c = __popc(w & 0xffu);
  if (r >= c) { r -= c; w >>= 8; base += 8; }
  c = __popc(w & 0xfu);
  if (r >= c) { r -= c; w >>= 4; base += 4; }
  c = __popc(w & 0x3u);
  if (r >= c) { r -= c; w >>= 2; base += 2; }
  return base + (r >= (int)(w & 1u) ? 1 : 0);
}

constexpr int kSumWords = 1024;  // summary bits: bitmaps up to 1024 * 32 words (2^20 values)

// Exclusive prefix over the block (one value per thread, kBigThreads
// threads); returns the prefix and leaves the total in *total.
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* s_tmp, int64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) s_tmp[warp] = incl;
  __syncthreads();
  int64_t wpre = 0, tot = 0;
  for (int w = 0; w < (kBigThreads >> 5); ++w) {
    const int64_t t = s_tmp[w];
    wpre += w < warp ? t : 0;
    tot += t;
  }
  *total = tot;
  __syncthreads();  // s_tmp may be reused right after
  return wpre + incl - v;
}

// Long rows (> kWarpRowCap entries): one CTA per row, rows taken from a
// work counter longest first.  A row holds distinct node ids (a canonical
// pair is visited once), so it is ordered through a two-level bitmap over
// its value range [min, max]: one bit per value (in shared memory when the
// range fits kBlockRowCap words, else in this CTA's global bitmap) and one
// summary bit per non-empty bitmap word.  The summary gives the non-empty
// words in order (written over the row's raw entries, which are no longer
// needed), and warps then walk chunks of 32 such words, finding the q-th
// set bit for q = lane, lane + 32, ... so the output writes are coalesced.
// The cost is O(n + range / 1024) per row, and only the words that were set
// are cleared again.  Repeated entries (seen when a bit was already set) or
// ranges beyond the summary send the row to a bitonic network instead (in
// shared memory up to kBlockRowCap entries, else in place in global memory).
__global__ void __launch_bounds__(kBigThreads, 3)
    k_rows_big(const int32_t* __restrict__ big_rows, uint32_t* __restrict__ n_big,
               int64_t list_cap, RowTable ta, RowTable tb, int index_bits,
               uint32_t* __restrict__ bitmaps, int64_t universe) {
  extern __shared__ uint32_t s_dyn[];  // kBlockRowCap words: bitmap, or a row to sort
  __shared__ uint32_t s_sum[kSumWords];
  __shared__ int32_t s_cc[kSumWords];  // per-chunk counts, then bases (< n < 2^31)
  __shared__ int64_t s_tmp[32];
  __shared__ int32_t s_min[32], s_max[32];
  __shared__ uint32_t s_item;
  __shared__ int s_dup;
  const uint32_t n_long = n_big[0], n_mid = n_big[8];
  const int64_t gwords = (universe + 31) / 32;
  uint32_t* gbm = bitmaps + (int64_t)blockIdx.x * gwords;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = nt >> 5;
  for (int w = tid; w < kBlockRowCap; w += nt) s_dyn[w] = 0u;
  for (int w = tid; w < kSumWords; w += nt) s_sum[w] = 0u;
  if (gwords > kBlockRowCap)
    for (int64_t w = tid; w < gwords; w += nt) gbm[w] = 0u;
  __syncthreads();
  __shared__ RowTable s_tab;  // the current row's table (picked by thread 0)
  __shared__ int32_t s_row;
  while (true) {
    if (tid == 0) {
      const uint32_t bb = atomicAdd(&n_big[9], 1u);
      s_item = bb;
      s_dup = 0;
      if (bb < n_long + n_mid) {
        const int32_t g = bb < n_long ? big_rows[bb] : big_rows[list_cap - 1 - (bb - n_long)];
        const bool second = g >= ta.rows;
        s_tab = second ? tb : ta;
        s_row = second ? g - (int32_t)ta.rows : g;
      }
    }
    __syncthreads();
    const uint32_t b = s_item;
    if (b >= n_long + n_mid) break;
    const RowTable& T = s_tab;
    const int32_t r = s_row;
    const int64_t* __restrict__ row_off = T.off;
    const int32_t* __restrict__ row_cnt = T.cnt;
    const int32_t* __restrict__ row_level = T.lvl;
    int32_t* __restrict__ raw = T.raw;
    const int64_t* __restrict__ raw_off = T.roff;
    const int32_t* __restrict__ row_base = T.rbase;
    void* vals_out = T.vals;
    void* tgt_out = T.tgts;
    void* lvl_out = T.lvls;
    const int64_t off = row_off[r];
    const int64_t roff = raw_off ? raw_off[r] : off;  // where the raw row is read
    const int32_t vbase = row_base ? row_base[r] : 0;   // ids written relative to it
    const int64_t n = row_cnt[r];
    const int32_t lvl = row_level ? row_level[r] : 0;
    // eight loads in flight per thread: a long row is otherwise a chain of
    // dependent global round trips
    constexpr int kU = 8;
    int32_t vmin = INT32_MAX, vmax = INT32_MIN;
    for (int64_t k = tid; k < n; k += (int64_t)nt * kU) {
      int32_t v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int64_t kk = k + (int64_t)u * nt;
        v[u] = kk < n ? raw[roff + kk] : INT32_MAX;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        if (k + (int64_t)u * nt < n) {
          vmin = v[u] < vmin ? v[u] : vmin;
          vmax = v[u] > vmax ? v[u] : vmax;
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vmin = min(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
      vmax = max(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    }
    if (lane == 0) {
      s_min[warp] = vmin;
      s_max[warp] = vmax;
    }
    __syncthreads();
    vmin = s_min[0];
    vmax = s_max[0];
    for (int w = 1; w < nwarps; ++w) {
      vmin = min(vmin, s_min[w]);
      vmax = max(vmax, s_max[w]);
    }
    const int64_t words = ((int64_t)vmax - vmin + 1 + 31) >> 5;
    const int64_t swords = (words + 31) >> 5;
    bool sorted = false;
    if (swords <= kSumWords) {
      uint32_t* bm = words <= kBlockRowCap ? s_dyn : gbm;
      bool dup = false;
      const bool dense = n >= 8 * words;
      // trip count shared by the lanes of a warp (the loop body votes)
      for (int64_t k = tid; k - lane < n; k += (int64_t)nt * kU) {
        int32_t w[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const int64_t kk = k + (int64_t)u * nt;
          w[u] = kk < n ? raw[roff + kk] : 0;
        }
        // Dense rows (at least 8 ids per bitmap word on average, e.g. the
        // near rows of halo leaves) have their ids in clustered runs, so the
        // lanes of a warp mostly set bits of the same word: one atomic per
        // word group (the group's bits ORed first; a repeated id shows as
        // fewer bits than lanes or as a bit already set), and the summary
        // is built by ballots afterwards.  Sparse rows set their bits and
        // summary bits directly.
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const bool valid = k + (int64_t)u * nt < n;
          if (dense) {
            const unsigned act = __ballot_sync(0xffffffffu, valid);
            if (valid) {
              const uint32_t v = (uint32_t)(w[u] - vmin);
              const uint32_t bit = 1u << (v & 31);
              const unsigned peers = __match_any_sync(act, v >> 5);
              const unsigned comb = __reduce_or_sync(peers, bit);
              if (lane == __ffs(peers) - 1) {
                const uint32_t old = atomicOr(&bm[v >> 5], comb);
                if ((old & comb) != 0u || __popc(comb) != __popc(peers)) dup = true;
              }
            }
          } else if (valid) {
            const uint32_t v = (uint32_t)(w[u] - vmin);
            const uint32_t bit = 1u << (v & 31);
            if (atomicOr(&bm[v >> 5], bit) & bit) dup = true;
            atomicOr(&s_sum[v >> 10], 1u << ((v >> 5) & 31));
          }
        }
      }
      if (dup) s_dup = 1;
      __syncthreads();
      if (dense && !s_dup) {
        for (int64_t w0 = (int64_t)warp * 32; w0 < words; w0 += (int64_t)nwarps * 32) {
          const int64_t ww = w0 + lane;
          const unsigned m = __ballot_sync(0xffffffffu, ww < words && bm[ww] != 0u);
          if (lane == 0) s_sum[w0 >> 5] = m;
        }
        __syncthreads();
      }
      if (s_dup) {
        // undo the bits; the row goes to the bitonic network
        for (int64_t k = tid; k < n; k += nt) {
          const uint32_t v = (uint32_t)(raw[roff + k] - vmin);
          bm[v >> 5] = 0u;
        }
        for (int64_t w = tid; w < swords; w += nt) s_sum[w] = 0u;
        __syncthreads();
      } else {
        // Non-empty words in ascending order -> raw[roff, roff + m).
        constexpr int kSumPer = kSumWords / kBigThreads;
        int64_t c = 0;
#pragma unroll
        for (int k = 0; k < kSumPer; ++k) {
          const int64_t sw = (int64_t)tid * kSumPer + k;
          c += sw < swords ? __popc(s_sum[sw]) : 0;
        }
        int64_t m;
        int64_t base = block_excl_scan(c, s_tmp, &m);
#pragma unroll
        for (int k = 0; k < kSumPer; ++k) {
          const int64_t sw = (int64_t)tid * kSumPer + k;
          uint32_t bits = sw < swords ? s_sum[sw] : 0u;
          while (bits) {
            const int bit = __ffs(bits) - 1;
            bits &= bits - 1;
            raw[roff + base++] = (int32_t)(sw * 32 + bit);
          }
        }
        __syncthreads();
        // bits per chunk of 32 listed words
        const int64_t nch = (m + 31) >> 5;
        for (int64_t ch = warp; ch < nch; ch += nwarps) {
          const int64_t j = ch * 32 + lane;
          int cnt = j < m ? __popc(bm[raw[roff + j]]) : 0;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
          if (lane == 0) s_cc[ch] = cnt;
        }
        __syncthreads();
        {
          int64_t cv[kSumPer];
          int64_t mine = 0;
#pragma unroll
          for (int k = 0; k < kSumPer; ++k) {
            const int64_t ch = (int64_t)tid * kSumPer + k;
            cv[k] = ch < nch ? s_cc[ch] : 0;
            mine += cv[k];
          }
          int64_t tot;
          int64_t run = block_excl_scan(mine, s_tmp, &tot);
#pragma unroll
          for (int k = 0; k < kSumPer; ++k) {
            const int64_t ch = (int64_t)tid * kSumPer + k;
            if (ch < nch) s_cc[ch] = (int32_t)run;
            run += cv[k];
          }
        }
        __syncthreads();
        for (int64_t ch = warp; ch < nch; ch += nwarps) {
          const int64_t j = ch * 32 + lane;
          const int32_t wi = j < m ? raw[roff + j] : 0;
          const uint32_t word = j < m ? bm[wi] : 0u;
          const int c1 = __popc(word);
          int incl = c1;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
          }
          const int T = __shfl_sync(0xffffffffu, incl, 31);
          const int64_t pos = off + s_cc[ch];
          for (int q0 = 0; q0 < T; q0 += 32) {
            const int q = q0 + lane;
            // lo = listed words whose inclusive count is <= q (lo <= 31)
            int lo = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
              const int v = __shfl_sync(0xffffffffu, incl, lo + step - 1);
              if (v <= q) lo += step;
            }
            const uint32_t wsel = __shfl_sync(0xffffffffu, word, lo);
            const int ex = __shfl_sync(0xffffffffu, incl - c1, lo);
            const int32_t wsi = __shfl_sync(0xffffffffu, wi, lo);
            if (q < T) {
              const int32_t v = vmin + wsi * 32 + select_bit(wsel, q - ex);
              store_idx(vals_out, index_bits, pos + q, v - vbase);
              if (tgt_out) {
                store_idx(tgt_out, index_bits, pos + q, r - vbase);
                store_idx(lvl_out, index_bits, pos + q, lvl);
              }
            }
          }
        }
        __syncthreads();
        for (int64_t j = tid; j < m; j += nt) bm[raw[roff + j]] = 0u;
        for (int64_t w = tid; w < swords; w += nt) s_sum[w] = 0u;
        __syncthreads();
        sorted = true;
      }
    }
    if (!sorted) {
      if (n <= kBlockRowCap) {
        int32_t* a = reinterpret_cast<int32_t*>(s_dyn);
        for (int64_t k = tid; k < n; k += nt) a[k] = raw[roff + k];
        __syncthreads();
        mirrored_bitonic<true>(a, n, tid, nt);
        emit_row(a, n, off, index_bits, vals_out, tgt_out, lvl_out, r - vbase, vbase, lvl, tid, nt);
        __syncthreads();
        for (int64_t k = tid; k < n; k += nt) s_dyn[k] = 0u;  // bitmap stays zero
      } else {
        int32_t* a = raw + roff;
        mirrored_bitonic<true>(a, n, tid, nt);
        emit_row(a, n, off, index_bits, vals_out, tgt_out, lvl_out, r - vbase, vbase, lvl, tid, nt);
      }
    }
    __syncthreads();
  }
}

// Dense neighbour leaf positions (L x max_nbr) of _result_to_neighbors.
__global__ void k_neighbor_leaf_positions(const int64_t* __restrict__ near_off,
                                          const int32_t* __restrict__ near_cnt, int64_t L,
                                          const void* neighbors, int index_bits,
                                          const int32_t* __restrict__ leafpos, int64_t max_nbr,
                                          void* out) {
  const int64_t total = L * max_nbr;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / max_nbr, k = e - j * max_nbr;
    int64_t v = -1;
    if (k < near_cnt[j]) v = leafpos[load_idx(neighbors, index_bits, near_off[j] + k)];
    store_idx(out, index_bits, e, v);
  }
}

}  // namespace

struct TravScratch {
  uint32_t* status;
  unsigned long long* stats;
  uint32_t* sizes;  // per generation
  uint32_t* n_big;
  NodeRec* recs;
  int32_t* far_cnt;
  int32_t* near_cnt;
  int32_t* cnt_by_level;
  int64_t* obl;
  int64_t* far_off;
  int64_t* near_off;
  unsigned long long* far_pos;
  unsigned long long* near_pos;
  int64_t* scan_tmp;
  int32_t* big_rows;
  int32_t* class_rows;  // kRowClasses lists of total + L rows
  uint32_t* bitmaps;
  int2* wf[2];
  uint32_t* region_cnt[2];
  unsigned long long* log_cnt;
  int2* log;
  unsigned long long log_region;
  // predicted mode
  int64_t* pad_far;   // total + 1
  int64_t* pad_near;  // L + 1
  unsigned long long* end_far;
  unsigned long long* end_near;
  int32_t* ext_far_cnt;
  int32_t* ext_near_cnt;
  int64_t* ext_far_off;   // total + 1
  int64_t* ext_near_off;  // L + 1
  int64_t* raw_off_far;
  int64_t* raw_off_near;
  int64_t* raw_end_far;
  int64_t* raw_end_near;
};

constexpr int kMaxGens = 4096;
// Every CTA of a generation appends at most 4 x kWalkThreads pairs per input
// chunk; a region of at least that size keeps small walks from overflowing.
constexpr int64_t kMinRegion = 4 * kWalkThreads;
static int64_t region_capacity(int64_t cap) {
  const int64_t r = cap / kWalkGrid;
  return r < kMinRegion ? kMinRegion : r;
}
constexpr int kBigGrid = kNumSMs * 3;

RowSortScratch carve_row_sort(Arena& a, int64_t total, int64_t L) {
  RowSortScratch s;
  s.stride = total + L;
  s.n_big = a.take<uint32_t>(64);
  s.big_rows = a.take<int32_t>(s.stride);
  s.class_rows = a.take<int32_t>((size_t)kRowClasses * s.stride);
  s.bitmaps = a.take<uint32_t>((size_t)kBigGrid * ((total + 31) / 32));
  return s;
}

int row_sort_pass(const RowSortScratch& s, const RowTable& a, const RowTable& b, int index_bits,
                  int64_t universe, cudaStream_t stream) {
  const int grid_small = kNumSMs * g_tune.row_grid_per_sm;
  const size_t big_smem = sizeof(int32_t) * kBlockRowCap;
  static std::atomic<uint64_t> big_attr{0};
  if (ensure_smem_limit(k_rows_big, (int)big_smem, big_attr) != cudaSuccess) return YGX_ERR_CUDA;
  const int64_t rows = a.rows + b.rows;
  if (a.rows < 0 || b.rows < 0 || rows > s.stride || rows > INT32_MAX) return YGX_ERR_ARG;
  if (cudaMemsetAsync(s.n_big, 0, 16 * sizeof(uint32_t), stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  k_rows_classify<<<grid_for(rows, 256), 256, 0, stream>>>(a, b, s.class_rows, s.stride,
                                                           s.n_big + 1, s.big_rows, s.n_big);
  YGX_CHECK_LAUNCH();
#define YGX_ROWS(C, R)                                                                        \
  k_rows_class<R><<<grid_small, 256, 0, stream>>>(s.class_rows + (C) * s.stride,             \
                                                  s.n_big + 1 + (C), a, b, index_bits);       \
  YGX_CHECK_LAUNCH();
  YGX_ROWS(0, 1) YGX_ROWS(1, 2) YGX_ROWS(2, 4) YGX_ROWS(3, 8) YGX_ROWS(4, 16) YGX_ROWS(5, 32)
#undef YGX_ROWS
  k_rows_big<<<kBigGrid, kBigThreads, big_smem, stream>>>(s.big_rows, s.n_big, s.stride, a, b,
                                                          index_bits, s.bitmaps, universe);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

// Entries per CTA log region for a total log capacity.
static int64_t log_region_capacity(int64_t log_cap) {
  const int64_t r = (log_cap + kWalkGrid - 1) / kWalkGrid;
  return r < 1 ? 1 : r;
}

static TravScratch carve_trav(Arena& a, int64_t total, int64_t L, int64_t cap, int64_t log_cap) {
  TravScratch s;
  s.status = a.take<uint32_t>(64);
  s.stats = a.take<unsigned long long>(kStatWords);
  s.sizes = a.take<uint32_t>(kMaxGens + 2);
  // [0] rows > kBlockRowCap, [1..6] class counts, [8] other long rows, [9] work counter
  s.n_big = a.take<uint32_t>(64);
  s.recs = a.take<NodeRec>(total);
  s.far_cnt = a.take<int32_t>(total);
  s.near_cnt = a.take<int32_t>(L);
  s.cnt_by_level = a.take<int32_t>(total);
  s.obl = a.take<int64_t>(total + 1);
  s.far_off = a.take<int64_t>(total + 1);
  s.near_off = a.take<int64_t>(L + 1);
  // one cursor array: far rows 0..total-1, then the near rows
  s.far_pos = a.take<unsigned long long>(total + L);
  s.near_pos = s.far_pos ? s.far_pos + total : nullptr;
  s.scan_tmp = a.take<int64_t>(scan_scratch_elems(total > L ? total : L));
  s.big_rows = a.take<int32_t>(total + L);  // far and near rows sort in one pass
  s.class_rows = a.take<int32_t>((size_t)kRowClasses * (total + L));
  s.bitmaps = a.take<uint32_t>((size_t)kBigGrid * ((total + 31) / 32));
  s.wf[0] = a.take<int2>(region_capacity(cap) * kWalkGrid);
  s.wf[1] = a.take<int2>(region_capacity(cap) * kWalkGrid);
  s.region_cnt[0] = a.take<uint32_t>(kWalkGrid);
  s.region_cnt[1] = a.take<uint32_t>(kWalkGrid);
  s.log_cnt = a.take<unsigned long long>(kWalkGrid);
  s.log_region = (unsigned long long)log_region_capacity(log_cap);
  s.log = a.take<int2>((size_t)s.log_region * kWalkGrid);
  s.pad_far = a.take<int64_t>(total + 1);
  s.pad_near = a.take<int64_t>(L + 1);
  s.end_far = a.take<unsigned long long>(total);
  s.end_near = a.take<unsigned long long>(L);
  s.ext_far_cnt = a.take<int32_t>(total);
  s.ext_near_cnt = a.take<int32_t>(L);
  s.ext_far_off = a.take<int64_t>(total + 1);
  s.ext_near_off = a.take<int64_t>(L + 1);
  s.raw_off_far = a.take<int64_t>(total);
  s.raw_off_near = a.take<int64_t>(L);
  s.raw_end_far = a.take<int64_t>(total);
  s.raw_end_near = a.take<int64_t>(L);
  return s;
}

// CTAs of every walk generation: a knob, at most kWalkGrid (the number of
// wavefront / log regions the workspace holds; regions past the grid stay
// empty).
static int walk_grid() {
  int b = g_tune.walk_blocks_per_sm;
  b = b < 1 ? 1 : (b > kWalkBlocksPerSM ? kWalkBlocksPerSM : b);
  return kNumSMs * b;
}

static int launch_gen(int mode, int mac, const TravScratch& s, int32_t ni, int32_t total_nodes,
                      float theta_sq, float theta, int gen, uint32_t cap, const RowSink& sink,
                      cudaStream_t st) {
  const int2* in = s.wf[gen & 1];
  int2* out = s.wf[(gen + 1) & 1];
  const uint32_t* cin = s.region_cnt[gen & 1];
  uint32_t* cout = s.region_cnt[(gen + 1) & 1];
  const uint32_t R = (uint32_t)region_capacity(cap);
#define YGX_GEN(MODE, MAC)                                                                  \
  k_walk_gen<MODE, MAC><<<walk_grid(), kWalkThreads, 0, st>>>(                              \
      s.recs, ni, total_nodes, theta_sq, theta, in, out, cin, cout, R, s.sizes, gen,        \
      s.far_cnt, s.near_cnt, s.log, s.log_cnt, s.log_region, sink, s.stats, s.status)
#define YGX_GEN_MAC(MODE)                     \
  if (mac == kMacBH) YGX_GEN(MODE, kMacBH);   \
  else if (mac == kMacDehnen) YGX_GEN(MODE, kMacDehnen); \
  else YGX_GEN(MODE, kMacEngblom);
  switch (mode) {
    case kWalkLog: YGX_GEN_MAC(kWalkLog) break;
    case kWalkCount: YGX_GEN_MAC(kWalkCount) break;
    case kWalkFill: YGX_GEN_MAC(kWalkFill) break;
    case kWalkPred: YGX_GEN_MAC(kWalkPred) break;
    default: return YGX_ERR_ARG;
  }
#undef YGX_GEN_MAC
#undef YGX_GEN
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

// Seeds (root, root) and launches the generations.  With fixed_gens < 0 the
// wavefront size is probed every 16 generations until it is empty (or a
// wavefront overflow is flagged); otherwise exactly fixed_gens generations
// run (a repeat of a walk whose length is known).  *gens_out = launched.
// The roots: one (root) or a forest (leaf_off != nullptr).
struct Roots {
  int root;
  const int64_t* leaf_off;
  int64_t S;
  const int32_t* parent32;
  const uint32_t* seg_flags;
};

static int run_gens(int mode, int mac, const TravScratch& s, int32_t ni, int32_t total,
                    float theta_sq, float theta_r, const Roots& roots, uint32_t cap,
                    const RowSink& sink, int fixed_gens, int gens_hint, int* gens_out,
                    cudaStream_t stream) {
  if (roots.leaf_off)
    k_seed_forest<<<1, 256, 0, stream>>>(s.wf[0], s.region_cnt[0], s.sizes,
                                         (uint32_t)region_capacity(cap), walk_grid(),
                                         roots.leaf_off,
                                         roots.S, roots.parent32, roots.seg_flags, s.status);
  else
    k_seed<<<1, 256, 0, stream>>>(s.wf[0], s.region_cnt[0], s.sizes, roots.root);
  YGX_CHECK_LAUNCH();
  int gen = 0, rc = YGX_OK;
  if (fixed_gens >= 0) {
    for (; gen < fixed_gens; ++gen) {
      rc = launch_gen(mode, mac, s, ni, total, theta_sq, theta_r, gen, cap, sink, stream);
      if (rc) return rc;
    }
    *gens_out = gen;
    return YGX_OK;
  }
  // The first probe comes after gens_hint generations (the length of a
  // previous walk of the same kind, so usually the only probe), later ones
  // every 16.
  int chunk = gens_hint > 0 ? gens_hint : 16;
  while (true) {
    for (int k = 0; k < chunk && gen < kMaxGens; ++k, ++gen) {
      rc = launch_gen(mode, mac, s, ni, total, theta_sq, theta_r, gen, cap, sink, stream);
      if (rc) return rc;
    }
    chunk = 16;
    uint32_t probe = 0, flags = 0;
    if (cudaMemcpyAsync(&probe, s.sizes + gen, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                        stream) != cudaSuccess ||
        cudaMemcpyAsync(&flags, s.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return YGX_ERR_CUDA;
    // A wavefront overflow ends the walk at once; a log overflow does not
    // (the walk goes on counting, so the log need it reports is exact).
    if (probe == 0 || (flags & ~(uint32_t)kFlagLogOverflow) != 0) break;
    if (gen >= kMaxGens) {
      *gens_out = gen;
      return YGX_ERR_QUEUE_OVERFLOW;
    }
  }
  *gens_out = gen;
  return YGX_OK;
}

// Row offsets from the counts in the workspace: level-major far offsets and
// the index-dtype offset / count tables, leaf-order near offsets.
static int row_offsets(const TravScratch& s, int64_t total, int64_t L, const int32_t* nbl32,
                       const void* tree_level_offsets, int num_levels, int index_bits,
                       void* node_offsets, void* far_counts, void* level_offsets,
                       void* near_offsets, void* near_counts, cudaStream_t stream) {
  k_gather_counts<<<grid_for(total, 256), 256, 0, stream>>>(s.far_cnt, nbl32, total,
                                                            s.cnt_by_level);
  YGX_CHECK_LAUNCH();
  int rc = exclusive_scan<int32_t>(s.cnt_by_level, total, s.obl, s.scan_tmp, stream);
  if (rc) return rc;
  k_far_offsets<<<grid_for(total + 1, 256), 256, 0, stream>>>(
      s.obl, nbl32, s.far_cnt, total, index_bits, s.far_off, node_offsets, far_counts,
      tree_level_offsets, num_levels, level_offsets);
  YGX_CHECK_LAUNCH();
  rc = exclusive_scan<int32_t>(s.near_cnt, L, s.near_off, s.scan_tmp, stream);
  if (rc) return rc;
  k_near_offsets<<<grid_for(L + 1, 256), 256, 0, stream>>>(s.near_off, s.near_cnt, L,
                                                           index_bits, near_offsets, near_counts);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

static RowSink no_sink() {
  RowSink k;
  k.far_pos = k.near_pos = nullptr;
  k.far_end = k.near_end = nullptr;
  k.far_src = k.near_nbr = nullptr;
  k.far_total = k.near_total = 0;
  return k;
}

}  // namespace ygx

extern "C" {

size_t ygx_traverse_workspace_size(int64_t total, int64_t num_leaves, int64_t wf_capacity,
                                   int64_t log_capacity) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_trav(a, total, num_leaves, wf_capacity, log_capacity);
  return a.used + 256;
}

static int trav_setup(ygx::TravScratch& s, void* ws, size_t ws_bytes, int64_t total, int64_t L,
                      int64_t cap, int64_t log_cap) {
  if (cap < 4 || cap > (int64_t)UINT32_MAX - 4096 || log_cap < 1) return YGX_ERR_ARG;
  if (ws_bytes < ygx_traverse_workspace_size(total, L, cap, log_cap)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  s = ygx::carve_trav(a, total, L, cap, log_cap);
  return YGX_OK;
}

// The walk.  Builds the per-node walk records (center + MAC extent +
// children + leaf position), walks from (root, root) generation by
// generation until the wavefront is empty (checked every 16 generations),
// counting every far / near row entry and logging every accepted / near
// pair, and copies to the host: stats_out[YGX_TSTAT_WORDS] (far/near totals
// and maxima, decision counters, max wavefront, generations, and the
// wavefront / log capacities that would have fit) and the status flags.
// leafpos32[node] is the near-row position of a leaf (-1 for internal
// nodes).  Synchronizes the stream.
static int walk_impl(const float* center, const float* radius, const float* max_extent,
                     const int32_t* left32, const int32_t* right32, const int32_t* leafpos32,
                     int64_t total, int64_t num_internal, int mac, float theta,
                     float dehnen_radius_scale, const ygx::Roots& roots, int mode, int gens_hint,
                     int64_t wf_capacity, int64_t log_capacity, uint64_t* stats_out,
                     uint32_t* flags_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
  const int64_t L = total - num_internal;
  ygx::TravScratch s;
  int rc = trav_setup(s, ws, ws_bytes, total, L, wf_capacity, log_capacity);
  if (rc) return rc;
  // theta^2 in fp32 (jnp.asarray(theta, float32) ** 2) and its sqrt.
  const float th = theta;
  const float theta_sq = th * th;
  const float theta_r = sqrtf(theta_sq);
  if (cudaMemsetAsync(s.status, 0, (char*)(s.n_big + 64) - (char*)s.status, stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  if (cudaMemsetAsync(s.far_cnt, 0, sizeof(int32_t) * total, stream) != cudaSuccess ||
      cudaMemsetAsync(s.near_cnt, 0, sizeof(int32_t) * L, stream) != cudaSuccess ||
      cudaMemsetAsync(s.log_cnt, 0, sizeof(unsigned long long) * ygx::kWalkGrid, stream) !=
          cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_node_recs<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      center, radius, max_extent, left32, right32, leafpos32, total, mac, dehnen_radius_scale,
      s.recs, s.status);
  YGX_CHECK_LAUNCH();
  int gen = 0;
  rc = ygx::run_gens(mode == YGX_WALK_LOG ? ygx::kWalkLog : ygx::kWalkCount, mac, s,
                     (int32_t)num_internal, (int32_t)total, theta_sq, theta_r, roots,
                     (uint32_t)wf_capacity, ygx::no_sink(), -1, gens_hint, &gen, stream);
  if (rc == YGX_ERR_QUEUE_OVERFLOW) flags_out[0] = ygx::kFlagQueueOverflow;
  if (rc) return rc;
  ygx::k_count_stats<<<ygx::grid_for(total, 256, ygx::kNumSMs * 4), 256, 0, stream>>>(
      s.far_cnt, total, s.near_cnt, L, s.sizes, gen, s.log_cnt, s.stats);
  YGX_CHECK_LAUNCH();
  if (cudaMemcpyAsync(stats_out, s.stats, sizeof(uint64_t) * YGX_TSTAT_WORDS,
                      cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(flags_out, s.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}

int ygx_traverse_walk(const float* center, const float* radius, const float* max_extent,
                      const int32_t* left32, const int32_t* right32, const int32_t* leafpos32,
                      int64_t total, int64_t num_internal, int mac, float theta,
                      float dehnen_radius_scale, int root, int mode, int gens_hint,
                      int64_t wf_capacity, int64_t log_capacity, uint64_t* stats_out,
                      uint32_t* flags_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 3 || total > INT32_MAX || num_internal < 1 || mac < 0 || mac > 2 ||
      root < 0 || root >= total || !stats_out || !flags_out ||
      (mode != YGX_WALK_LOG && mode != YGX_WALK_COUNT))
    return YGX_ERR_ARG;
  return walk_impl(center, radius, max_extent, left32, right32, leafpos32, total, num_internal,
                   mac, theta, dehnen_radius_scale, ygx::Roots{root, nullptr, 0, nullptr, nullptr},
                   mode, gens_hint, wf_capacity, log_capacity, stats_out, flags_out, ws, ws_bytes,
                   stream);
}

// The walk over a forest of S trees (ygx_batch_build_topology: set s at
// nodes 2 leaf_off[s] - s, leafpos32 / left32 / right32 / parent32 with
// global ids), all sets in one wavefront from (root_s, root_s); the
// counts, pair log and stats as ygx_traverse_walk (YGX_WALK_LOG mode), so
// ygx_traverse_fill / ygx_traverse_finalize follow on the same workspace
// with total = all nodes and num_internal = total_leaves - S.
int ygx_batch_traverse_walk(const float* center, const float* radius, const float* max_extent,
                            const int32_t* left32, const int32_t* right32,
                            const int32_t* leafpos32, const int32_t* parent32, int64_t total,
                            const int64_t* leaf_off, int64_t S, const uint32_t* seg_flags,
                            int mac, float theta, float dehnen_radius_scale, int gens_hint,
                            int64_t wf_capacity, int64_t log_capacity, uint64_t* stats_out,
                            uint32_t* flags_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 1 || total > INT32_MAX || S < 1 || !leaf_off || !parent32 || mac < 0 || mac > 2 ||
      !stats_out || !flags_out)
    return YGX_ERR_ARG;
  const int64_t total_leaves = (total + S) / 2;
  return walk_impl(center, radius, max_extent, left32, right32, leafpos32, total,
                   total_leaves - S, mac, theta, dehnen_radius_scale,
                   ygx::Roots{0, leaf_off, S, parent32, seg_flags}, YGX_WALK_LOG, gens_hint,
                   wf_capacity, log_capacity, stats_out, flags_out, ws, ws_bytes, stream);
}

// Fill (after a walk without overflow on the same workspace).  Writes the
// level-major far layout and the near CSR: node_offsets (total+1),
// far_counts (total), level_offsets (num_levels+1), near_offsets (L+1),
// near_counts (L) in the index dtype, and the raw rows far_src32 (far
// total) / near_nbr32 (near total) in log order.  Does not synchronize.
int ygx_traverse_fill(int64_t total, int64_t num_internal, int64_t wf_capacity,
                      int64_t log_capacity, int64_t far_total, int64_t near_total,
                      const int32_t* nbl32, const int32_t* leafpos32,
                      const void* tree_level_offsets, int num_levels, int index_bits,
                      void* node_offsets, void* far_counts, void* level_offsets,
                      void* near_offsets, void* near_counts, int32_t* far_src32,
                      int32_t* near_nbr32, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 3 || total > INT32_MAX || num_internal < 1 || far_total < 0 || near_total < 0 ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  const int64_t L = total - num_internal;
  ygx::TravScratch s;
  int rc = trav_setup(s, ws, ws_bytes, total, L, wf_capacity, log_capacity);
  if (rc) return rc;
  rc = ygx::row_offsets(s, total, L, nbl32, tree_level_offsets, num_levels, index_bits,
                        node_offsets, far_counts, level_offsets, near_offsets, near_counts,
                        stream);
  if (rc) return rc;
  ygx::k_init_cursors<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.far_off, total, s.far_pos,
                                                                     s.near_off, L, s.near_pos);
  YGX_CHECK_LAUNCH();
  ygx::k_log_scatter<<<ygx::kWalkGrid, 256, 0, stream>>>(
      s.log, s.log_cnt, s.log_region, leafpos32, (int32_t)total, s.far_pos,
      (unsigned long long)far_total, (unsigned long long)near_total, far_src32, near_nbr32,
      s.status, 0u);
  YGX_CHECK_LAUNCH();
  ygx::k_check_cursors<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      s.far_off, s.far_cnt, s.far_pos, total, s.near_off, s.near_cnt, s.near_pos, L, s.status);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

// Second walk of the plain two-pass mode (after ygx_traverse_walk with
// YGX_WALK_COUNT on the same workspace): the offset tables as in
// ygx_traverse_fill, then the same `gens` generations again, each directed
// entry written at its row's atomic cursor, and every cursor checked
// against its row end.  Does not synchronize.
int ygx_traverse_fill_walk(int64_t total, int64_t num_internal, int mac, float theta, int root,
                           int64_t wf_capacity, int64_t log_capacity, int gens,
                           int64_t far_total, int64_t near_total, const int32_t* nbl32,
                           const void* tree_level_offsets, int num_levels, int index_bits,
                           void* node_offsets, void* far_counts, void* level_offsets,
                           void* near_offsets, void* near_counts, int32_t* far_src32,
                           int32_t* near_nbr32, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 3 || total > INT32_MAX || num_internal < 1 || mac < 0 || mac > 2 || root < 0 ||
      root >= total || gens < 0 || gens > ygx::kMaxGens || far_total < 0 || near_total < 0 ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  const int64_t L = total - num_internal;
  ygx::TravScratch s;
  int rc = trav_setup(s, ws, ws_bytes, total, L, wf_capacity, log_capacity);
  if (rc) return rc;
  const float th = theta;
  const float theta_sq = th * th;
  const float theta_r = sqrtf(theta_sq);
  rc = ygx::row_offsets(s, total, L, nbl32, tree_level_offsets, num_levels, index_bits,
                        node_offsets, far_counts, level_offsets, near_offsets, near_counts,
                        stream);
  if (rc) return rc;
  if (cudaMemsetAsync(s.sizes, 0, sizeof(uint32_t) * (ygx::kMaxGens + 2), stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_init_cursors<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.far_off, total, s.far_pos,
                                                                     s.near_off, L, s.near_pos);
  YGX_CHECK_LAUNCH();
  ygx::RowSink sink = ygx::no_sink();
  sink.far_pos = s.far_pos;
  sink.near_pos = s.near_pos;
  sink.far_src = far_src32;
  sink.near_nbr = near_nbr32;
  sink.far_total = (unsigned long long)far_total;
  sink.near_total = (unsigned long long)near_total;
  int ran = 0;
  rc = ygx::run_gens(ygx::kWalkFill, mac, s, (int32_t)num_internal, (int32_t)total, theta_sq,
                     theta_r, ygx::Roots{root, nullptr, 0, nullptr, nullptr},
                     (uint32_t)wf_capacity, sink, gens, 0, &ran, stream);
  if (rc) return rc;
  ygx::k_check_cursors<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      s.far_off, s.far_cnt, s.far_pos, total, s.near_off, s.near_cnt, s.near_pos, L, s.status);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

// ---- predicted (learned one-pass) mode ---------------------------------------

// Padded row offsets from predicted capacities (far_cap32[node],
// near_cap32[leaf position]) into the workspace; sums_out (host, 2 words)
// gets the padded totals, which the raw row buffers must hold at least.
// Synchronizes the stream.
int ygx_traverse_pad_offsets(int64_t total, int64_t num_internal, int64_t wf_capacity,
                             int64_t log_capacity, const int32_t* far_cap32,
                             const int32_t* near_cap32, uint64_t* sums_out, void* ws,
                             size_t ws_bytes, cudaStream_t stream) {
  if (total < 3 || num_internal < 1 || !far_cap32 || !near_cap32 || !sums_out) return YGX_ERR_ARG;
  const int64_t L = total - num_internal;
  ygx::TravScratch s;
  int rc = trav_setup(s, ws, ws_bytes, total, L, wf_capacity, log_capacity);
  if (rc) return rc;
  if ((rc = ygx::exclusive_scan<int32_t>(far_cap32, total, s.pad_far, s.scan_tmp, stream)))
    return rc;
  if ((rc = ygx::exclusive_scan<int32_t>(near_cap32, L, s.pad_near, s.scan_tmp, stream)))
    return rc;
  int64_t sums[2];
  if (cudaMemcpyAsync(&sums[0], s.pad_far + total, sizeof(int64_t), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaMemcpyAsync(&sums[1], s.pad_near + L, sizeof(int64_t), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  sums_out[0] = (uint64_t)sums[0];
  sums_out[1] = (uint64_t)sums[1];
  return YGX_OK;
}

// One-pass walk into the padded rows set up by ygx_traverse_pad_offsets on
// the same workspace (far_cap32 / near_cap32 are the same capacities).
// Entries past a row's capacity go to the pair log.  Afterwards the
// workspace holds the exact row lengths; stats_out adds YGX_TSTAT_OVF_ROWS /
// _OVF_ENTRIES (rows that outgrew their capacity, entries past it) and
// _EXT_FAR / _EXT_NEAR (extension space ygx_traverse_fill_predicted needs
// beyond the padded totals).  Flags as in ygx_traverse_walk.  Synchronizes.
int ygx_traverse_walk_predicted(const float* center, const float* radius,
                                const float* max_extent, const int32_t* left32,
                                const int32_t* right32, const int32_t* leafpos32, int64_t total,
                                int64_t num_internal, int mac, float theta,
                                float dehnen_radius_scale, int root, int gens_hint,
                                int64_t wf_capacity, int64_t log_capacity,
                                const int32_t* far_cap32,
                                const int32_t* near_cap32, int32_t* far_raw32,
                                int32_t* near_raw32, uint64_t* stats_out, uint32_t* flags_out,
                                void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 3 || 2 * total > INT32_MAX || num_internal < 1 || mac < 0 || mac > 2 || root < 0 ||
      root >= total || !far_cap32 || !near_cap32 || !far_raw32 || !near_raw32 || !stats_out ||
      !flags_out)
    return YGX_ERR_ARG;
  const int64_t L = total - num_internal;
  ygx::TravScratch s;
  int rc = trav_setup(s, ws, ws_bytes, total, L, wf_capacity, log_capacity);
  if (rc) return rc;
  const float th = theta;
  const float theta_sq = th * th;
  const float theta_r = sqrtf(theta_sq);
  if (cudaMemsetAsync(s.status, 0, (char*)(s.n_big + 64) - (char*)s.status, stream) !=
          cudaSuccess ||
      cudaMemsetAsync(s.log_cnt, 0, sizeof(unsigned long long) * ygx::kWalkGrid, stream) !=
          cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_node_recs<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      center, radius, max_extent, left32, right32, leafpos32, total, mac, dehnen_radius_scale,
      s.recs, s.status);
  YGX_CHECK_LAUNCH();
  ygx::k_pad_ends<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.pad_far, far_cap32, total,
                                                                 s.end_far, s.far_pos);
  YGX_CHECK_LAUNCH();
  ygx::k_pad_ends<<<ygx::grid_for(L, 256), 256, 0, stream>>>(s.pad_near, near_cap32, L,
                                                             s.end_near, s.near_pos);
  YGX_CHECK_LAUNCH();
  ygx::RowSink sink = ygx::no_sink();
  sink.far_pos = s.far_pos;
  sink.near_pos = s.near_pos;
  sink.far_end = s.end_far;
  sink.near_end = s.end_near;
  sink.far_src = far_raw32;
  sink.near_nbr = near_raw32;
  int gen = 0;
  rc = ygx::run_gens(ygx::kWalkPred, mac, s, (int32_t)num_internal, (int32_t)total, theta_sq,
                     theta_r, ygx::Roots{root, nullptr, 0, nullptr, nullptr},
                     (uint32_t)wf_capacity, sink, -1, gens_hint, &gen, stream);
  if (rc == YGX_ERR_QUEUE_OVERFLOW) flags_out[0] = ygx::kFlagQueueOverflow;
  if (rc) return rc;
  ygx::k_pred_counts<<<ygx::grid_for(total, 256, ygx::kNumSMs * 4), 256, 0, stream>>>(
      s.far_pos, s.pad_far, far_cap32, total, s.far_cnt, s.ext_far_cnt, s.stats,
      ygx::kStatExtFar);
  YGX_CHECK_LAUNCH();
  ygx::k_pred_counts<<<ygx::grid_for(L, 256, ygx::kNumSMs * 4), 256, 0, stream>>>(
      s.near_pos, s.pad_near, near_cap32, L, s.near_cnt, s.ext_near_cnt, s.stats,
      ygx::kStatExtNear);
  YGX_CHECK_LAUNCH();
  ygx::k_count_stats<<<ygx::grid_for(total, 256, ygx::kNumSMs * 4), 256, 0, stream>>>(
      s.far_cnt, total, s.near_cnt, L, s.sizes, gen, s.log_cnt, s.stats);
  YGX_CHECK_LAUNCH();
  if (cudaMemcpyAsync(stats_out, s.stats, sizeof(uint64_t) * YGX_TSTAT_WORDS,
                      cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(flags_out, s.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}

// After ygx_traverse_walk_predicted without overflow flags: the offset
// tables as in ygx_traverse_fill; rows that outgrew their capacity moved to
// the extension area behind the padded rows (raw buffers of far_raw_cap /
// near_raw_cap entries, at least padded total + YGX_TSTAT_EXT_*) and
// completed from the log; far_raw_off / near_raw_off (device int64 per row)
// receive where each raw row starts, for ygx_traverse_finalize.  Does not
// synchronize.
int ygx_traverse_fill_predicted(int64_t total, int64_t num_internal, int64_t wf_capacity,
                                int64_t log_capacity, const int32_t* far_cap32,
                                const int32_t* near_cap32, int64_t far_raw_cap,
                                int64_t near_raw_cap, const int32_t* nbl32,
                                const void* tree_level_offsets, int num_levels, int index_bits,
                                void* node_offsets, void* far_counts, void* level_offsets,
                                void* near_offsets, void* near_counts, int32_t* far_raw32,
                                int32_t* near_raw32, int64_t* far_raw_off, int64_t* near_raw_off,
                                void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 3 || 2 * total > INT32_MAX || num_internal < 1 || !far_cap32 || !near_cap32 ||
      !far_raw32 || !near_raw32 || !far_raw_off || !near_raw_off ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  const int64_t L = total - num_internal;
  ygx::TravScratch s;
  int rc = trav_setup(s, ws, ws_bytes, total, L, wf_capacity, log_capacity);
  if (rc) return rc;
  rc = ygx::row_offsets(s, total, L, nbl32, tree_level_offsets, num_levels, index_bits,
                        node_offsets, far_counts, level_offsets, near_offsets, near_counts,
                        stream);
  if (rc) return rc;
  if ((rc = ygx::exclusive_scan<int32_t>(s.ext_far_cnt, total, s.ext_far_off, s.scan_tmp, stream)))
    return rc;
  if ((rc = ygx::exclusive_scan<int32_t>(s.ext_near_cnt, L, s.ext_near_off, s.scan_tmp, stream)))
    return rc;
  // moved-row lists: far rows in big_rows, near rows in class_rows (both
  // hold at least max(total, L) entries and are free until the finalize); counters
  // in n_big[10] / n_big[11]
  if (cudaMemsetAsync(s.n_big + 10, 0, 2 * sizeof(uint32_t), stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_relocate_mark<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      s.pad_far, far_cap32, s.ext_far_cnt, s.ext_far_off, total, far_raw_cap, s.far_pos,
      s.raw_off_far, s.big_rows, s.n_big + 10, s.status, ygx::kFlagFarOverflow);
  YGX_CHECK_LAUNCH();
  ygx::k_relocate_mark<<<ygx::grid_for(L, 256), 256, 0, stream>>>(
      s.pad_near, near_cap32, s.ext_near_cnt, s.ext_near_off, L, near_raw_cap, s.near_pos,
      s.raw_off_near, s.class_rows, s.n_big + 11, s.status, ygx::kFlagNearOverflow);
  YGX_CHECK_LAUNCH();
  ygx::k_relocate_copy<<<ygx::kNumSMs * 8, 256, 0, stream>>>(s.big_rows, s.n_big + 10, s.pad_far,
                                                            far_cap32, s.raw_off_far, far_raw32);
  YGX_CHECK_LAUNCH();
  ygx::k_relocate_copy<<<ygx::kNumSMs * 8, 256, 0, stream>>>(
      s.class_rows, s.n_big + 11, s.pad_near, near_cap32, s.raw_off_near, near_raw32);
  YGX_CHECK_LAUNCH();
  ygx::k_raw_ends<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.raw_off_far, s.far_cnt, total,
                                                                 s.raw_end_far);
  YGX_CHECK_LAUNCH();
  ygx::k_raw_ends<<<ygx::grid_for(L, 256), 256, 0, stream>>>(s.raw_off_near, s.near_cnt, L,
                                                             s.raw_end_near);
  YGX_CHECK_LAUNCH();
  ygx::k_ovf_scatter<<<ygx::kWalkGrid, 256, 0, stream>>>(
      s.log, s.log_cnt, s.log_region, (int32_t)total, s.far_pos, s.near_pos, far_raw32,
      near_raw32, s.raw_end_far, s.raw_end_near, s.status);
  YGX_CHECK_LAUNCH();
  ygx::k_check_ext<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      s.far_pos, s.raw_end_far, s.ext_far_cnt, total, s.status, ygx::kFlagFarOverflow);
  YGX_CHECK_LAUNCH();
  ygx::k_check_ext<<<ygx::grid_for(L, 256), 256, 0, stream>>>(
      s.near_pos, s.raw_end_near, s.ext_near_cnt, L, s.status, ygx::kFlagNearOverflow);
  YGX_CHECK_LAUNCH();
  if (cudaMemcpyAsync(far_raw_off, s.raw_off_far, sizeof(int64_t) * total,
                      cudaMemcpyDeviceToDevice, stream) != cudaSuccess ||
      cudaMemcpyAsync(near_raw_off, s.raw_off_near, sizeof(int64_t) * L,
                      cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}

// Finalize: canonical (ascending) order within every row, widened into the
// index-dtype outputs: far sources / targets / target_levels in the
// level-major layout, near neighbours in leaf order.  far_src32 and
// near_nbr32 are sorted in place for rows longer than 8192.  If
// neighbor_leaf_positions is non-null it receives the dense (L x max_nbr)
// leaf-position table.  Does not synchronize.
static int finalize_impl(const ygx::TravScratch& s, int64_t total, int64_t L,
                         const int32_t* level32, const int32_t* leafpos32, int index_bits,
                         int32_t* far_src32, int32_t* near_nbr32, const int64_t* far_raw_off,
                         const int64_t* near_raw_off, const int32_t* far_row_base,
                         const int32_t* near_row_base, void* far_sources, void* far_targets,
                         void* target_levels, void* neighbors, void* neighbor_leaf_positions,
                         int64_t max_nbr, cudaStream_t stream);

int ygx_traverse_finalize(int64_t total, int64_t num_internal, int64_t wf_capacity,
                          int64_t log_capacity, const int32_t* level32, const int32_t* leafpos32,
                          int index_bits, int32_t* far_src32, int32_t* near_nbr32,
                          const int64_t* far_raw_off, const int64_t* near_raw_off,
                          const int32_t* far_row_base, const int32_t* near_row_base,
                          void* far_sources,
                          void* far_targets, void* target_levels, void* neighbors,
                          void* neighbor_leaf_positions, int64_t max_nbr, void* ws,
                          size_t ws_bytes, cudaStream_t stream) {
  if (total < 3 || num_internal < 1 || (index_bits != 32 && index_bits != 64)) return YGX_ERR_ARG;
  const int64_t L = total - num_internal;
  ygx::TravScratch s;
  int rc = trav_setup(s, ws, ws_bytes, total, L, wf_capacity, log_capacity);
  if (rc) return rc;
  return finalize_impl(s, total, L, level32, leafpos32, index_bits, far_src32, near_nbr32,
                       far_raw_off, near_raw_off, far_row_base, near_row_base, far_sources,
                       far_targets, target_levels, neighbors, neighbor_leaf_positions, max_nbr,
                       stream);
}

static int finalize_impl(const ygx::TravScratch& s, int64_t total, int64_t L,
                         const int32_t* level32, const int32_t* leafpos32, int index_bits,
                         int32_t* far_src32, int32_t* near_nbr32, const int64_t* far_raw_off,
                         const int64_t* near_raw_off, const int32_t* far_row_base,
                         const int32_t* near_row_base, void* far_sources, void* far_targets,
                         void* target_levels, void* neighbors, void* neighbor_leaf_positions,
                         int64_t max_nbr, cudaStream_t stream) {
  const ygx::RowSortScratch rs{s.n_big, s.big_rows, s.class_rows, s.bitmaps, total + L};
  const ygx::RowTable far_rows{total, s.far_off, s.far_cnt, level32, far_src32, far_raw_off,
                               far_row_base, far_sources, far_targets, target_levels};
  const ygx::RowTable near_rows{L, s.near_off, s.near_cnt, nullptr, near_nbr32, near_raw_off,
                                near_row_base, neighbors, nullptr, nullptr};
  const int rc2 = ygx::row_sort_pass(rs, far_rows, near_rows, index_bits, total, stream);
  if (rc2) return rc2;
  if (neighbor_leaf_positions && max_nbr > 0) {
    ygx::k_neighbor_leaf_positions<<<ygx::grid_for(L * max_nbr, 256), 256, 0, stream>>>(
        s.near_off, s.near_cnt, L, neighbors, index_bits, leafpos32, max_nbr,
        neighbor_leaf_positions);
    YGX_CHECK_LAUNCH();
  }
  return YGX_OK;
}

int ygx_traverse_status(const void* ws, uint32_t* flags_out, cudaStream_t stream) {
  return ygx_status_read(ws, flags_out, stream);
}

// The batched walk, fill and finalize of ygx_batch_traverse_walk +
// ygx_traverse_fill + ygx_traverse_finalize in one call that never
// synchronizes or copies to the host, so it can be captured in a CUDA graph
// and replayed: every size is the caller's -- exactly `gens` walk
// generations, the wavefront / log capacities, and far_capacity /
// near_capacity entries in the output lists (far_src32 / sources / targets /
// target_levels hold far_capacity, near_nbr32 / neighbors near_capacity).
// A walk that does not fit (wavefront left after the last generation, a
// wavefront or log region overflow, totals above the capacities) sets its
// flag in the workspace status word and the lists are left unwritten (all
// row counts zero); ygx_traverse_stats_read afterwards returns the flags and
// the statistics (totals, generations, the capacities that would have
// fitted), from which the caller re-sizes.  Rows are written with node ids
// local to each set (minus node_base32 / leaf_base32).  No reference
// counterpart (the reference builds one tree per call and sizes on the
// host).
int ygx_batch_traverse_lists(
    const float* center, const float* radius, const float* max_extent, const int32_t* left32,
    const int32_t* right32, const int32_t* leafpos32, const int32_t* parent32,
    const int32_t* nbl32, const int32_t* level32, const int32_t* node_base32,
    const int32_t* leaf_base32, int64_t total, const int64_t* leaf_off, int64_t S,
    const uint32_t* seg_flags, int mac, float theta, float dehnen_radius_scale, int gens,
    int64_t wf_capacity, int64_t log_capacity, int64_t far_capacity, int64_t near_capacity,
    int index_bits, void* node_offsets, void* far_counts, void* near_offsets, void* near_counts,
    int32_t* far_src32, int32_t* near_nbr32, void* sources, void* targets, void* target_levels,
    void* neighbors, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 3 || total > INT32_MAX || S < 1 || !leaf_off || !parent32 || mac < 0 || mac > 2 ||
      gens < 1 || gens > ygx::kMaxGens || far_capacity < 1 || near_capacity < 1 ||
      (index_bits != 32 && index_bits != 64) || !far_src32 || !near_nbr32 || !sources ||
      !targets || !target_levels || !neighbors)
    return YGX_ERR_ARG;
  const int64_t Lt = (total + S) / 2, ni = Lt - S;
  if (ni < 1 || 2 * Lt - S != total) return YGX_ERR_ARG;
  ygx::TravScratch s;
  int rc = trav_setup(s, ws, ws_bytes, total, Lt, wf_capacity, log_capacity);
  if (rc) return rc;
  const float th = theta;
  const float theta_sq = th * th;
  const float theta_r = sqrtf(theta_sq);
  if (cudaMemsetAsync(s.status, 0, (char*)(s.n_big + 64) - (char*)s.status, stream) != cudaSuccess ||
      cudaMemsetAsync(s.far_cnt, 0, sizeof(int32_t) * total, stream) != cudaSuccess ||
      cudaMemsetAsync(s.near_cnt, 0, sizeof(int32_t) * Lt, stream) != cudaSuccess ||
      cudaMemsetAsync(s.log_cnt, 0, sizeof(unsigned long long) * ygx::kWalkGrid, stream) !=
          cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_node_recs<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      center, radius, max_extent, left32, right32, leafpos32, total, mac, dehnen_radius_scale,
      s.recs, s.status);
  YGX_CHECK_LAUNCH();
  int ran = 0;
  rc = ygx::run_gens(ygx::kWalkLog, mac, s, (int32_t)ni, (int32_t)total, theta_sq, theta_r,
                     ygx::Roots{0, leaf_off, S, parent32, seg_flags}, (uint32_t)wf_capacity,
                     ygx::no_sink(), gens, 0, &ran, stream);
  if (rc) return rc;
  ygx::k_count_stats<<<ygx::grid_for(total, 256, ygx::kNumSMs * 4), 256, 0, stream>>>(
      s.far_cnt, total, s.near_cnt, Lt, s.sizes, gens, s.log_cnt, s.stats);
  YGX_CHECK_LAUNCH();
  ygx::k_guard_totals<<<1, 32, 0, stream>>>(s.sizes, gens, s.stats,
                                            (unsigned long long)far_capacity,
                                            (unsigned long long)near_capacity, s.status);
  YGX_CHECK_LAUNCH();
  const uint32_t stop = ygx::kFlagQueueOverflow | ygx::kFlagLogOverflow | ygx::kFlagFarOverflow |
                        ygx::kFlagNearOverflow | ygx::kFlagBadInput | ygx::kFlagTimeout;
  ygx::k_zero_counts_if<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.status, stop, s.far_cnt,
                                                                       total, s.near_cnt, Lt);
  YGX_CHECK_LAUNCH();
  rc = ygx::row_offsets(s, total, Lt, nbl32, nullptr, -1, index_bits, node_offsets, far_counts,
                        nullptr, near_offsets, near_counts, stream);
  if (rc) return rc;
  ygx::k_init_cursors<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.far_off, total, s.far_pos,
                                                                     s.near_off, Lt, s.near_pos);
  YGX_CHECK_LAUNCH();
  ygx::k_log_scatter<<<ygx::kWalkGrid, 256, 0, stream>>>(
      s.log, s.log_cnt, s.log_region, leafpos32, (int32_t)total, s.far_pos,
      (unsigned long long)far_capacity, (unsigned long long)near_capacity, far_src32, near_nbr32,
      s.status, stop);
  YGX_CHECK_LAUNCH();
  ygx::k_check_cursors<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      s.far_off, s.far_cnt, s.far_pos, total, s.near_off, s.near_cnt, s.near_pos, Lt, s.status);
  YGX_CHECK_LAUNCH();
  return finalize_impl(s, total, Lt, level32, leafpos32, index_bits, far_src32, near_nbr32,
                       nullptr, nullptr, node_base32, leaf_base32, sources, targets,
                       target_levels, neighbors, nullptr, 0, stream);
}

// Copies the statistics words (YGX_TSTAT_*) and the status flags of a
// traversal workspace to the host; synchronizes the stream.
int ygx_traverse_stats_read(int64_t total, int64_t num_leaves, int64_t wf_capacity,
                            int64_t log_capacity, const void* ws, size_t ws_bytes,
                            uint64_t* stats_out, uint32_t* flags_out, cudaStream_t stream) {
  if (!stats_out || !flags_out) return YGX_ERR_ARG;
  ygx::TravScratch s;
  int rc = trav_setup(s, const_cast<void*>(ws), ws_bytes, total, num_leaves, wf_capacity,
                      log_capacity);
  if (rc) return rc;
  if (cudaMemcpyAsync(stats_out, s.stats, sizeof(uint64_t) * YGX_TSTAT_WORDS,
                      cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(flags_out, s.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}

}  // extern "C"
