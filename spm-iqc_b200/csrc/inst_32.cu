// Kernel chains for the 32^3 grid (FP64 and FP32).
#include "ops_impl.cuh"

const OpsTable *spm_table_32(int prec) {
  return prec == 0 ? spm::Impl<32, double>::table() : spm::Impl<32, float>::table();
}
