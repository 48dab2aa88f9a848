/*
 * Test infrastructure (oracle) -- never product code.
 *
 * The oracle restatement (hamr_oracle.c) compiled with every double a
 * forward-mode dual number (dual_prelude.hpp): liboracle_dual.so, whose
 * arrays hold (value, tangent) pairs. Used by the adjoint tests as an FP64
 * tangent-linear reference independent of the CUDA library's hand-written
 * reverse sweep.
 */
#include "dual_prelude.hpp"
extern "C" {
#include "hamr_oracle.c"
}
