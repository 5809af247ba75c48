// One expansion order of the pass kernels (built once per order with -DJB_ORDER=P).
#include "fmm_adjoint.cuh"

#ifndef JB_ORDER
#error "JB_ORDER must be defined"
#endif

template struct jb::RunP2M<JB_ORDER>;
template struct jb::RunM2M<JB_ORDER>;
template struct jb::RunM2L<JB_ORDER>;
template struct jb::RunM2LMixed<JB_ORDER>;
template struct jb::RunL2L<JB_ORDER>;
template struct jb::RunL2LLeaves<JB_ORDER>;
template struct jb::RunLeafEval<JB_ORDER>;
template struct jb::RunTargets<JB_ORDER>;
#if JB_ORDER <= 9
template struct jb::RunAdj<JB_ORDER>;
#endif
