// Host harness that runs the reference's 6-worker codelet `MultiSWAffine`
// (src/codelets/codelet_multi_affine.cpp) on the CPU, workers one after the
// other.  Same build and use rules as codelet_batch_harness.cpp.
#define private public
#include "codelets/codelet_multi_affine.cpp"
#undef private
#define REF_VERTEX MultiSWAffine
#define REF_PREFIX ref_codelet_multi
#define REF_MULTI 1
#include "harness_common.inc"
