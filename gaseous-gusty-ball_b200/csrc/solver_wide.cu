// solver_wide.cu — the 640-thread solve kernels (grids from N = 384 on, where
// more loads in flight per SM shorten the staged phases), compiled in their
// own translation unit from the same device code as solver.cu's 512-thread
// kernels (solver_body.cuh), so that neither kernel's inlining and register
// allocation depends on the other's.
#include <algorithm>
#include <cstdio>
#include <type_traits>
#include <vector>

#include "ggb_internal.h"
#include "ggb_solver.h"

namespace ggb {
namespace wide {

#include "solver_body.cuh"

}  // namespace wide

const void *pcg_wide_kernel(bool mixed) {
    return mixed ? (const void *)wide::k_pcg<true, wide::kPBWide> : (const void *)wide::k_pcg<false, wide::kPBWide>;
}

void pcg_wide_trace_symbols(void **trace_n, void **stage_trace, void **stage_n, void **stage_all) {
    GGB_CHECK(cudaGetSymbolAddress(trace_n, wide::g_trace_n));
    GGB_CHECK(cudaGetSymbolAddress(stage_trace, wide::g_stage_trace));
    GGB_CHECK(cudaGetSymbolAddress(stage_n, wide::g_stage_trace_n));
    GGB_CHECK(cudaGetSymbolAddress(stage_all, wide::g_stage_trace_all));
}

}  // namespace ggb
