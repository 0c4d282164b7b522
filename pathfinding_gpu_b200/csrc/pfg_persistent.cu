// pfg_persistent.cu - one group of instantiations of the persistent kernel,
// selected at compile time: PFG_V_ASTAR (0 / 1), PFG_V_AM (atomic mode 0..2),
// PFG_V_PART (0: Thread and Warp mappings, 1: Hybrid mapping, 2: Hybrid mapping
// with warp-worker drains, 3: Hybrid mapping with independent bucket windows, SSSP
// only). The build compiles this file once per group, in
// parallel, and pfg_kernels.cu reaches each group's kernels through its getter.
#include "pfg_persistent.cuh"

#if !defined(PFG_V_ASTAR) || !defined(PFG_V_AM) || !defined(PFG_V_PART)
#error "compile with -DPFG_V_ASTAR=.. -DPFG_V_AM=.. -DPFG_V_PART=.."
#endif

#define PFG_GETTER_NAME2(A, AM, P) persistent_kernel_##A##_##AM##_##P
#define PFG_GETTER_NAME(A, AM, P) PFG_GETTER_NAME2(A, AM, P)

namespace pfg {

const void* PFG_GETTER_NAME(PFG_V_ASTAR, PFG_V_AM, PFG_V_PART)(int map) {
    constexpr bool A = PFG_V_ASTAR != 0;
#if PFG_V_PART == 0
    return map == 0 ? (const void*)k_persistent<A, PFG_V_AM, 0> : (const void*)k_persistent<A, PFG_V_AM, 1>;
#elif PFG_V_PART == 1
    (void)map;
    return (const void*)k_persistent<A, PFG_V_AM, 2>;
#elif PFG_V_PART == 2
    (void)map;
    return (const void*)k_persistent<A, PFG_V_AM, 2, true>;
#else
    (void)map;
    static_assert(!A, "independent windows exist for SSSP only");
    return (const void*)k_persistent<false, PFG_V_AM, 2, false, true>;
#endif
}

}  // namespace pfg
