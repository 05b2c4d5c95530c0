// Field files and initial data.
//  * The reference's ASCII field format (src/File_Op.cpp:8-89): one real value
//    per line, printed "%.16e \n", row-major, blocks of k eigenvectors
//    concatenated; read back with "%lf".
//  * A binary checkpoint (no counterpart in the reference): a fixed header
//    (magic, version, grid and model parameters, step, field count) and the
//    raw doubles, with an FNV-1a checksum of the payload.
//  * The reference's initData reader (get_initial_value,
//    src/Initialization.cpp:242-339): a mode count n, then n records of four
//    integers (k0 k1 k2 amplitude); mode j sets u_F[k] = 0.1 * amplitude at
//    k_i = round(k_i / l * L) (negative indices wrapped), later records
//    overwriting earlier ones. Integers are read one after another like the
//    reference's fscanf("%d") loop; a file with fewer integers than 4n leaves
//    the missing ones 0.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/spmiqc.h"
#include "spm_internal.h"

namespace {

constexpr char kMagic[8] = {'S', 'P', 'M', 'I', 'Q', 'C', 'K', '1'};

struct CkHeader {
  char magic[8];
  uint32_t version;
  int32_t N;
  int32_t nfields;
  int32_t precision;
  double L, Tau, Gamma, dt;
  int64_t step;
  uint64_t count;     // doubles in the payload
  uint64_t checksum;  // FNV-1a over the payload bytes
};

uint64_t fnv1a(const void *data, size_t bytes) {
  const unsigned char *p = static_cast<const unsigned char *>(data);
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < bytes; i++) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

struct File {
  FILE *f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

}  // namespace

extern "C" int spm_save_field_txt(const char *path, const double *x, size_t count) {
  if (!path || (!x && count)) return spm_fail(SPM_ERR_ARG, "null argument");
  File fp;
  fp.f = std::fopen(path, "w");
  if (!fp.f) return spm_fail(SPM_ERR_ARG, "cannot open the field file for writing");
  for (size_t i = 0; i < count; i++)
    if (std::fprintf(fp.f, "%.16e \n", x[i]) < 0) return spm_fail(SPM_ERR_STATE, "write failed");
  if (std::fclose(fp.f) != 0) {
    fp.f = nullptr;
    return spm_fail(SPM_ERR_STATE, "write failed");
  }
  fp.f = nullptr;
  return SPM_OK;
}

extern "C" int spm_load_field_txt(const char *path, double *x, size_t count) {
  if (!path || (!x && count)) return spm_fail(SPM_ERR_ARG, "null argument");
  File fp;
  fp.f = std::fopen(path, "r");
  if (!fp.f) return spm_fail(SPM_ERR_ARG, "cannot open the field file");
  for (size_t i = 0; i < count; i++)
    if (std::fscanf(fp.f, "%lf", &x[i]) != 1) return spm_fail(SPM_ERR_STATE, "the field file has fewer values than expected");
  return SPM_OK;
}

extern "C" int spm_checkpoint_save(const char *path, const spm_checkpoint_info *info, const double *fields) {
  if (!path || !info || !fields || info->N <= 0 || info->nfields <= 0) return spm_fail(SPM_ERR_ARG, "bad argument");
  CkHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kMagic, 8);
  h.version = 1;
  h.N = info->N;
  h.nfields = info->nfields;
  h.precision = info->precision;
  h.L = info->L;
  h.Tau = info->Tau;
  h.Gamma = info->Gamma;
  h.dt = info->dt;
  h.step = info->step;
  h.count = (uint64_t)info->nfields * (uint64_t)info->N * info->N * info->N;
  h.checksum = fnv1a(fields, h.count * sizeof(double));
  // write to a temporary name, then rename, so a crash never leaves a torn file
  std::vector<char> tmp(std::strlen(path) + 5);
  std::snprintf(tmp.data(), tmp.size(), "%s.tmp", path);
  File fp;
  fp.f = std::fopen(tmp.data(), "wb");
  if (!fp.f) return spm_fail(SPM_ERR_ARG, "cannot open the checkpoint for writing");
  if (std::fwrite(&h, sizeof(h), 1, fp.f) != 1 || std::fwrite(fields, sizeof(double), h.count, fp.f) != h.count)
    return spm_fail(SPM_ERR_STATE, "checkpoint write failed");
  const int rc = std::fclose(fp.f);
  fp.f = nullptr;
  if (rc != 0 || std::rename(tmp.data(), path) != 0) return spm_fail(SPM_ERR_STATE, "checkpoint write failed");
  return SPM_OK;
}

extern "C" int spm_checkpoint_load(const char *path, spm_checkpoint_info *info, double *fields, size_t capacity) {
  if (!path || !info) return spm_fail(SPM_ERR_ARG, "null argument");
  File fp;
  fp.f = std::fopen(path, "rb");
  if (!fp.f) return spm_fail(SPM_ERR_ARG, "cannot open the checkpoint");
  CkHeader h;
  if (std::fread(&h, sizeof(h), 1, fp.f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != 1)
    return spm_fail(SPM_ERR_STATE, "not a checkpoint of this library");
  if (h.N <= 0 || h.nfields <= 0 || h.count != (uint64_t)h.nfields * (uint64_t)h.N * h.N * h.N)
    return spm_fail(SPM_ERR_STATE, "corrupt checkpoint header");
  info->N = h.N;
  info->nfields = h.nfields;
  info->precision = h.precision;
  info->L = h.L;
  info->Tau = h.Tau;
  info->Gamma = h.Gamma;
  info->dt = h.dt;
  info->step = h.step;
  if (!fields) return SPM_OK;  // header only
  if (capacity < h.count) return spm_fail(SPM_ERR_ARG, "the buffer is smaller than the checkpoint");
  if (std::fread(fields, sizeof(double), h.count, fp.f) != h.count)
    return spm_fail(SPM_ERR_STATE, "truncated checkpoint");
  if (fnv1a(fields, h.count * sizeof(double)) != h.checksum) return spm_fail(SPM_ERR_STATE, "checkpoint checksum mismatch");
  return SPM_OK;
}

extern "C" int spm_initdata_spectrum(const char *path, int N, double L, double l, double *full) {
  if (!path || !full || N <= 0 || !(l > 0)) return spm_fail(SPM_ERR_ARG, "bad argument");
  File fp;
  fp.f = std::fopen(path, "r");
  if (!fp.f) return spm_fail(SPM_ERR_ARG, "cannot open the initData file");
  const size_t n3 = (size_t)N * N * N;
  std::memset(full, 0, sizeof(double) * 2 * n3);
  int n = 0;
  if (std::fscanf(fp.f, "%d", &n) != 1 || n < 0) return spm_fail(SPM_ERR_STATE, "initData: no mode count");
  std::vector<int> rec((size_t)n * 4, 0);
  for (size_t i = 0; i < rec.size(); i++)
    if (std::fscanf(fp.f, "%d", &rec[i]) != 1) break;
  for (int i = 0; i < n; i++) {
    int k[3];
    for (int d = 0; d < 3; d++) {
      k[d] = (int)std::round((double)rec[4 * i + d] / l * L);
      if (k[d] < 0) k[d] += N;
      if (k[d] < 0 || k[d] >= N) return spm_fail(SPM_ERR_STATE, "initData: mode outside the grid");
    }
    full[2 * ((size_t)k[0] * N * N + (size_t)k[1] * N + k[2])] = rec[4 * i + 3] * 0.1;
  }
  return SPM_OK;
}

// phi = Re(my_ifft(u_F)) for the spectrum of an initData file: the Hermitian
// part of u_F (the reference keeps u_F as read; its anti-Hermitian part only
// feeds the imaginary parts of the reference's fields, which the real-valued
// updates never read), packed and inverse transformed on the device.
extern "C" int spm_initial_field(spm_ctx *c, const char *path, double l, void *phi) {
  if (!c || !path || !phi) return spm_fail(SPM_ERR_ARG, "null argument");
  const int N = c->N;
  const size_t n3 = (size_t)N * N * N;
  std::vector<double> u(2 * n3), h(2 * n3);
  int rc = spm_initdata_spectrum(path, N, c->L, l, u.data());
  if (rc != SPM_OK) return rc;
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++)
      for (int k = 0; k < N; k++) {
        const size_t a = ((size_t)i * N + j) * N + k;
        const size_t b = ((size_t)((N - i) % N) * N + (N - j) % N) * N + (N - k) % N;
        h[2 * a] = 0.5 * (u[2 * a] + u[2 * b]);
        h[2 * a + 1] = 0.5 * (u[2 * a + 1] - u[2 * b + 1]);
      }
  void *dfull = nullptr, *dspec = nullptr;
  cudaError_t e = cudaMalloc(&dfull, sizeof(double) * 2 * n3);
  if (e == cudaSuccess) e = cudaMalloc(&dspec, c->field_bytes);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dfull, h.data(), sizeof(double) * 2 * n3, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) rc = spm_fail_cuda(e, "initial field buffers");
  if (rc == SPM_OK) rc = spm_spectrum_from_full(c, (const double *)dfull, dspec);
  if (rc == SPM_OK) rc = spm_ifft(c, dspec, phi);
  if (rc == SPM_OK) {
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) rc = spm_fail_cuda(e, "initial field");
  }
  cudaFree(dfull);
  cudaFree(dspec);
  return rc;
}
