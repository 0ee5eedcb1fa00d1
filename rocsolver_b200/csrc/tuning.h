// tuning.h -- run-time kernel configuration table (written by rocsolver_b200/tune.py).
//
// Replaces the reference's compile-time tuning tables (library/src/include/ideal_sizes.hpp:
// 208-240 getrf block sizes and kernel switch points, :166-180 potrf;
// roclapack_getrf.hpp:17-166), which need a rebuild to change
// (docs/design/tuning.rst:20-31).  Here the choices live in a text table that the
// autotuner measures on the GPU and the library reads when the first handle is created:
//
//   getrf    <s|d|t> <m_max> <threads> <rows_per_thread> <panel_width> <chunk> <fold>
//   vbatched <s|d> <n_max> <threads> <rows_per_thread> <panel_width> <chunk> <fold> <ctas_per_sm>
//
// An entry applies to sizes up to m_max (n_max: the batch's largest order) above the
// previous entry of the same kind and precision (t = the FP32 LU with split-TF32 trailing
// updates).  chunk = trailing-update column chunk
// (multiple of 32; 0 = the default), fold = 1 folds each panel's row interchanges into the
// trailing update, fold = 2 (precision t only) runs the trailing update on the tcgen05
// tensor cores (operands in shared-memory descriptors, accumulators in TMEM) for the
// variants compiled with it, ctas_per_sm = resident CTAs the persistent kernel launches per SM
// (0 = as many as fit).  Entries naming a kernel variant that is not compiled, or one too
// small for the size, are ignored (the built-in choice applies).
#pragma once

#include <stddef.h>

namespace rsb {

struct LuCfg
{
    int nt, r, jb, cw, fold;
};
struct VbCfg
{
    int nt, r, jb, cw, fold, per_sm;
};

// entry for (precision 's'/'d'/'t', size); false when the table has none
bool tuned_getrf(char prec, int m, LuCfg* out);
bool tuned_vbatched(char prec, int max_n, VbCfg* out);
// load the table named by ROCSOLVER_B200_TUNING, else tuning_b200.txt beside the library
// (once per process; later calls do nothing)
void tuning_load_default_once();

} // namespace rsb
