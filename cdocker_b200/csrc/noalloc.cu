// noalloc.cu -- a search entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc while they search: real-time loops that
// must not hit the allocator (cudaMalloc and cudaFree can synchronise the whole device and
// take unbounded time), and hosts whose device memory is owned by a pool or arena that
// forbids outside allocations. cdk_search_device grows its wave and table scratch with
// cudaMalloc on demand; cdk_search_device_noalloc runs the same FP32-form kernels with all of
// that scratch carved from one file-scope device array of fixed size instead.
//
// Limits and sharing rules:
//  * FP32-form contexts only. The tensor-core forms need an operator image that the context
//    builds with cudaMalloc on first use; a precision-form context is rejected with
//    CDK_ERR_UNSUPPORTED instead of silently searching in another form.
//  * g_noalloc_scratch is CDK_NOALLOC_SCRATCH_BYTES (64 MiB). Every GPU that loads this
//    library holds it until the process exits. A call splits its rotations into waves that
//    fit the array; a search whose single rotation does not fit (very large grid x ligand
//    box) is rejected with CDK_ERR_UNSUPPORTED.
//  * Host code cannot use the array's name as a device address. The first call on each
//    device, with that device current, looks the address up with cudaGetSymbolAddress and
//    caches it for the life of the process. The cache does not survive cudaDeviceReset (or
//    any teardown of the device's primary context): do not call this entry point after one.
//  * The call synchronises its stream twice: to read back the ligand-box plan and, at the
//    end, the overflow count.
//  * All calls share the array and it keeps the previous call's contents. The counters the
//    search relies on are cleared at the start of every call; everything else is written
//    before it is read. Calls that overlap on the GPU (two streams, two host threads) race on
//    the array: serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/cdock_b200.h"
#include "cdk_internal.h"

namespace cdk {
namespace {

constexpr size_t kScratchBytes = CDK_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// per-device address of the static array (set up once per device, device current)
int scratch_for_device(int dev, void** out) {
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal out of range for the no-alloc scratch");
    return CDK_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
      return CDK_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return CDK_OK;
}

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// misc words at the head of the array: [0] diameter bits, [1] input flags, [2] overflow
// count, [4..7] work counters (two u64)
constexpr size_t kMiscBytes = 256;

__global__ void k_na_check(int nAtom, int nConf, const float* coor, const int* slot, int K,
                           unsigned int* misc) {
  const long total = (long)nConf * nAtom * nAtom;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long c = t / ((long)nAtom * nAtom);
    const int i = (int)((t / nAtom) % nAtom), j = (int)(t % nAtom);
    if (j <= i) continue;
    const float* a = coor + (c * nAtom + i) * 3;
    const float* b = coor + (c * nAtom + j) * 3;
    const double dx = (double)a[0] - b[0], dy = (double)a[1] - b[1], dz = (double)a[2] - b[2];
    atomicMax(misc, __float_as_uint((float)sqrt(dx * dx + dy * dy + dz * dz)));
  }
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < (long)nConf * nAtom * 3;
       t += (long)gridDim.x * blockDim.x) {
    if (t < nAtom && (slot[t] < 0 || slot[t] > K - 2)) atomicOr(misc + 1, 1u);
    if (!isfinite(coor[t])) atomicOr(misc + 1, 2u);
  }
}

// rotation descriptors of one wave [r0, r0 + nr) and the atom parameters
__global__ void k_na_tables(long r0, int nr, int nAtom, int nConf, int nQ, const float* quats,
                            const float* charge, const float* eps, const int* slot,
                            ConfDesc* confs, RotDesc* rots, AtomParam* params) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nr) {
    const long g = r0 + t;
    RotDesc d;
    for (int i = 0; i < 4; ++i) d.q[i] = quats[g * 4 + i];
    d.conf = (int)(g / nQ);
    d.out = (int)g;
    d.pad0 = d.pad1 = 0;
    rots[t] = d;
  }
  if (t < nConf) confs[t] = ConfDesc{(int)t * nAtom, 0, nAtom, 0};
  if (t < nAtom) params[t] = AtomParam{sqrtf(eps[t]), charge[t], slot[t], 0};
}

#define NA_CUDA(call)                                                      \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));       \
      return CDK_ERR_CUDA;                                                 \
    }                                                                      \
  } while (0)

}  // namespace
}  // namespace cdk

using namespace cdk;

extern "C" int cdk_search_device_noalloc(cdk_ctx* ctx, int nAtom, int nConf,
                                         const float* d_coor, const float* d_charge,
                                         const float* d_eps, const int* d_slot, int nQ,
                                         const float* d_quats, float* d_minE, int* d_idx,
                                         void* stream) {
  CtxView v;
  if (!ctx_view(ctx, &v) || !d_coor || !d_charge || !d_eps || !d_slot || !d_minE || !d_idx ||
      (nQ > 0 && !d_quats)) {
    set_error("null argument");
    return CDK_ERR_INVALID;
  }
  if (nAtom <= 0 || nConf <= 0 || nQ < 0 || nAtom > v.max_atoms) {
    set_error("nAtom must be in [1, max_atoms], nConf positive, nQ non-negative");
    return CDK_ERR_INVALID;
  }
  const long nRot = (long)nConf * nQ;
  if (nRot == 0) return CDK_OK;
  if (nRot > (1l << 31) / 4) {
    set_error("too many rotations in one call");
    return CDK_ERR_INVALID;
  }
  if (v.form != CDK_FORM_FP32) {
    set_error("cdk_search_device_noalloc runs the FP32 form only; this context uses a "
              "tensor-core form (use cdk_search_device)");
    return CDK_ERR_UNSUPPORTED;
  }
  NA_CUDA(cudaSetDevice(v.dev));
  void* base = nullptr;
  int rc = scratch_for_device(v.dev, &base);
  if (rc) return rc;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : v.stream;
  const int n = v.n, K = v.K;
  const size_t ncol = (size_t)n * (n / 2 + 1);
  char* p = static_cast<char*>(base);
  unsigned int* misc = reinterpret_cast<unsigned int*>(p);

  // inputs check and ligand box plan (one 8-byte read back)
  NA_CUDA(cudaMemsetAsync(misc, 0, kMiscBytes, s));
  {
    const long work = std::max<long>((long)nConf * nAtom * nAtom, (long)nConf * nAtom * 3);
    const long blocks = std::max<long>(1, std::min<long>(4096, (work + 255) / 256));
    k_na_check<<<(unsigned)blocks, 256, 0, s>>>(nAtom, nConf, d_coor, d_slot, K, misc);
    NA_CUDA(cudaGetLastError());
  }
  NA_CUDA(cudaMemcpyAsync(v.h_misc, misc, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  if (v.h_misc[1] & 1u) {
    set_error("atom slot outside [0, K-2]");
    return CDK_ERR_INVALID;
  }
  if (v.h_misc[1] & 2u) {
    set_error("non-finite ligand coordinate");
    return CDK_ERR_INVALID;
  }
  float diam;
  std::memcpy(&diam, &v.h_misc[0], sizeof(float));
  const int Lb = std::min(n, std::max(2, (int)std::floor(diam / v.spacing + 1e-3) + 3));

  // carve the array: misc | conf table | params | per-wave buffers
  const size_t b_conf = up256(sizeof(ConfDesc) * (size_t)nConf);
  const size_t b_par = up256(sizeof(AtomParam) * (size_t)nAtom);
  const size_t fixed = kMiscBytes + b_conf + b_par;
  const size_t per_rot = sizeof(RotDesc) + (size_t)nAtom * sizeof(float4) + sizeof(RotRec) +
                         sizeof(unsigned long long) + (size_t)K * Lb * ncol * sizeof(float2) +
                         (size_t)n * ncol * sizeof(float2);
  const size_t slack = 6 * 256;  // alignment of the six per-wave regions
  if (fixed + slack + per_rot > kScratchBytes) {
    set_error("search exceeds the no-alloc scratch (" + std::to_string(kScratchBytes >> 20) +
              " MiB): one rotation of this grid and ligand box needs " +
              std::to_string((fixed + slack + per_rot) >> 20) + " MiB; use cdk_search_device");
    return CDK_ERR_UNSUPPORTED;
  }
  int wave = (int)std::min<long>(nRot, (long)((kScratchBytes - fixed - slack) / per_rot));
  wave = std::min(wave, 65535);
  ConfDesc* confs = reinterpret_cast<ConfDesc*>(p + kMiscBytes);
  AtomParam* params = reinterpret_cast<AtomParam*>(p + kMiscBytes + b_conf);
  char* q = p + fixed;
  RotDesc* rots = reinterpret_cast<RotDesc*>(q);
  q += up256(sizeof(RotDesc) * (size_t)wave);
  WaveArgs a{};
  a.rot_xyz = reinterpret_cast<float4*>(q);
  q += up256((size_t)wave * nAtom * sizeof(float4));
  a.rec = reinterpret_cast<RotRec*>(q);
  q += up256((size_t)wave * sizeof(RotRec));
  a.keys = reinterpret_cast<unsigned long long*>(q);
  q += up256((size_t)wave * sizeof(unsigned long long));
  a.A = reinterpret_cast<float2*>(q);
  q += up256((size_t)wave * K * Lb * ncol * sizeof(float2));
  a.B = reinterpret_cast<float2*>(q);
  q += up256((size_t)wave * n * ncol * sizeof(float2));
  if ((size_t)(q - p) > kScratchBytes) {
    set_error("internal: no-alloc scratch layout overflow");
    return CDK_ERR_UNSUPPORTED;
  }
  a.n = n;
  a.K = K;
  a.Lb = Lb;
  a.spacing = v.spacing;
  a.max_atoms = nAtom;
  a.atom_cap = nAtom;
  a.coords = d_coor;
  a.params = params;
  a.confs = confs;
  a.phat = v.phat;
  a.tw = v.tw;
  a.minE = d_minE;
  a.idx = d_idx;
  a.err_count = reinterpret_cast<int*>(misc + 2);
  a.fault = reinterpret_cast<int*>(misc + 3);
  a.work = reinterpret_cast<unsigned long long*>(misc + 4);
  a.col_tile = v.col_tile_opt > 0 ? v.col_tile_opt : pick_col_tile(n, K);
  a.kyof = v.kyof;
  for (long r0 = 0; r0 < nRot; r0 += wave) {
    a.nrot = (int)std::min<long>(wave, nRot - r0);
    a.rots = rots;
    const long tmax = std::max<long>(a.nrot, std::max(nConf, nAtom));
    k_na_tables<<<(unsigned)((tmax + 255) / 256), 256, 0, s>>>(
        r0, a.nrot, nAtom, nConf, nQ, d_quats, d_charge, d_eps, d_slot, confs, rots, params);
    NA_CUDA(cudaGetLastError());
    NA_CUDA(launch_prep(a, s));
    NA_CUDA(launch_spread_yz(a, s));
    NA_CUDA(launch_xpass(a, s));
    NA_CUDA(launch_yz_inv_argmin(a, s));
    NA_CUDA(launch_finalize(a, s));
  }
  NA_CUDA(cudaMemcpyAsync(v.h_misc + 2, misc + 2, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  if (v.h_misc[2] != 0) {
    set_error(std::to_string(v.h_misc[2]) +
              " rotation(s) overflowed the planned ligand box; results for them are invalid");
    return CDK_ERR_OVERFLOW;
  }
  return CDK_OK;
}
