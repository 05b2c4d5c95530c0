// Kernel chains for the 160^3 grid (FP64 and FP32).
#include "ops_impl.cuh"

const OpsTable *spm_table_160(int prec) {
  return prec == 0 ? spm::Impl<160, double>::table() : spm::Impl<160, float>::table();
}
