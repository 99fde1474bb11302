// Host harness that runs the reference's own IPU codelet `SWAffine`
// (src/codelets/codelet_batch_affine.cpp) on the CPU.  The codelet source is
// compiled unmodified from the reference tree against the vertex-field
// stand-in in oracle/ref_shim.  Built by oracle/Makefile into oracle/_ref/.
// TEST INFRASTRUCTURE ONLY: used by tests, smoke() and bench.py's
// cpu_baseline/reference legs as the checker and the timed CPU reference.
#define private public  // the codelet keeps its C/bG scratch fields private
#include "codelets/codelet_batch_affine.cpp"
#undef private
#define REF_VERTEX SWAffine
#define REF_PREFIX ref_codelet_batch
#include "harness_common.inc"
