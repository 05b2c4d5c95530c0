// Kernel chains for the 256^3 grid (FP64 and FP32).
#include "ops_impl.cuh"

const OpsTable *spm_table_256(int prec) {
  return prec == 0 ? spm::Impl<256, double>::table() : spm::Impl<256, float>::table();
}
