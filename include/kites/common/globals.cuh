// globals.cuh -- enums and constants of the kites:: API (same names and
// values as farkhor/KiTES kites/common/globals.cuh:7-55, so user code that
// names them compiles unchanged).
#ifndef KITES_B200_GLOBALS_CUH_
#define KITES_B200_GLOBALS_CUH_

namespace kites {

enum {
  COMPILE_TIME_DETERMINED_BLOCK_SIZE = 128,
  WARP_SIZE = 32,
  WARP_SIZE_SHIFT = 5
};

// process<launch::async> runs like launch::sync (the reference's process
// template never reads its launch mode); copyMem<T, launch::async> enqueues
// its copy without waiting.
enum class launch { sync = true, async = false };
enum class operation_mode { iterative = true, frontier_based = false };
enum class input_graph_form { edge_list_s_d = true, edge_list_d_s = false };
enum class graph_property { directed = true, undirected = false };
enum class edge_list_expression { complete = true, incomplete = false };
enum class semi_dynamic_load_balancer { ON = true, OFF = false };

}  // namespace kites

#endif
