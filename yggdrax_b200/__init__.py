"""yggdrax_b200: the yggdrax tree pipeline on NVIDIA B200 (sm_100a).

Drop-in for yggdrax's tree-pipeline hot path -- Morton encode and stable
sort, radix/LBVH and fixed-depth builds with octree tables, node geometry,
and the symmetric dual-tree traversal -- with every stage running as
hand-written CUDA kernels from ``libygx.so`` (C ABI: ``include/ygx.h``).
Inputs and outputs are torch CUDA tensors in the reference's layouts.
"""

from .dtypes import INDEX_DTYPE, as_index
from .geometry import (LevelMajorTreeGeometry, TreeGeometry, compute_tree_geometry,
                       geometry_to_level_major)
from .interactions import (
    CompactTaggedFarPairs,
    DualTreeRetryEvent,
    DualTreeTraversalConfig,
    DualTreeWalkResult,
    MACType,
    NodeInteractionList,
    NodeNeighborList,
    build_compact_far_pairs,
    build_compact_far_pairs_and_leaf_neighbor_lists,
    build_interactions_and_neighbors,
    build_leaf_neighbor_lists,
    get_traversal_mode,
    set_default_dual_tree_config,
    set_dense_neighbor_budget,
    set_reference_limits,
    set_traversal_mode,
)
from .mutual import MutualWalkResult, dual_tree_walk_mutual
from .octree_walk import (CompactTaggedOctreeFarPairs, ExplicitOctreeBoxGeometry,
                          ExplicitOctreeTraversalView, OctreeNativeNeighborList,
                          build_explicit_octree_traversal_view, build_octree_native_far_pairs,
                          build_octree_native_neighbor_lists,
                          compute_explicit_octree_box_geometry)
from .tree_moments import (TreeMassMoments, TreeMultipoleMoments, compute_tree_mass_moments,
                           compute_tree_multipole_moments, pack_multipole_expansions)
from .dense_interactions import (DenseInteractionBuffers, build_dense_interactions,
                                 densify_interactions)
from .grouped_interactions import (GroupedInteractionBuffers, build_grouped_interactions,
                                   build_grouped_interactions_from_pairs)
from .morton import (
    encode_and_sort,
    get_common_prefix_length,
    infer_bounds,
    morton_encode,
    sort_by_morton,
)
from .tree import (
    MAX_TREE_LEVELS,
    FixedDepthTreeBuildConfig,
    OctreeTopology,
    OctreeTree,
    RadixTree,
    RadixTreeTopology,
    RadixTreeWorkspace,
    Tree,
    TreeBuildConfig,
    TreeBuilder,
    TreeBuildMode,
    TreeBuildRequest,
    TreeType,
    augment_radix_topology_with_octree,
    available_tree_types,
    build_explicit_octree_metadata,
    build_fixed_depth_octree,
    build_fixed_depth_octree_jit,
    build_fixed_depth_tree,
    build_fixed_depth_tree_jit,
    build_octree,
    build_octree_jit,
    build_tree,
    build_tree_jit,
    get_leaf_nodes,
    get_level_offsets,
    get_node_levels,
    get_nodes_by_level,
    get_num_internal_nodes,
    get_num_levels,
    register_tree_builder,
    resolve_tree_topology,
)

__all__ = [name for name in dir() if not name.startswith("_")]
