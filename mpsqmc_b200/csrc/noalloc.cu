// mpsqmc_local_energy_noalloc: the local-energy sweep of energy_kernel for callers that cannot
// allocate device memory.  All scratch lives in one file-scope device array (g_noalloc_scratch);
// the caller supplies the inputs and the output buffer.
//
// Array layout: per-CTA slices of [ compact-MPO environments | matrix work buffers, when they do
// not fit in shared memory ].  The bond-dimension tables travel as a kernel parameter, so a call
// issues no host-to-device copy.  The host never dereferences the array's name (in host code it
// is only a stand-in symbol): at the first call on a device, with that device current,
// cudaGetSymbolAddress gives the device address, which is kept per device and passed to the
// kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mpsqmc_gpu.h"

#define MQ_DEVICE_ONLY
#include "walker_kernels.cuh"

namespace mq_host {
void set_last_error(const std::string &msg);  // capi.cu: backs mpsqmc_last_error()
}

namespace {

constexpr int kMaxL = MPSQMC_NOALLOC_MAX_L;
constexpr size_t kScratchDoubles = MPSQMC_NOALLOC_SCRATCH_BYTES / sizeof(double);

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

struct Tables {
  int aT[kMaxL + 1];
  int bW[kMaxL + 1];
  long toff[kMaxL];
  long woff[kMaxL];
  double bondJ[kMaxL];
};

struct DeviceSetup {
  bool ready = false;
  double *scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int sm_count = 1;
  int smem_optin = 0;
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

// tab: the bond tables by value (a __grid_constant__ parameter, read in place).  big_off >= 0:
// the matrix work buffers sit at that offset of the CTA's slice instead of shared memory.
__global__ void __launch_bounds__(mq::kThreads, 1)
    energy_noalloc_kernel(mq::Dev p, const __grid_constant__ Tables tab, long big_off, const double *walkers,
                          long wstride, const double *ov, double *out, int N) {
  extern __shared__ double smem_raw[];
  mq::Smem s;
  double *slice = p.scratch + (long)blockIdx.x * p.scr_stride;
  mq::smem_doubles(p.L, p.maxA, p.maxB, p.G, p.pa, p.pb, p.pq, &s, smem_raw, big_off >= 0 ? slice + big_off : nullptr,
                   nullptr, false, false);
  const int L = p.L, tid = threadIdx.x;
  double *Fbuf = slice;
  const int fst = 4 * p.maxA * p.maxB;
  for (int w = blockIdx.x; w < N; w += gridDim.x) {
    const double *W = walkers + (long)w * wstride;
    if (tid == 0) s.Lenv[0] = 1.0;
    __syncthreads();
    int cur = 0;
    for (int k = 0; k < L; ++k) {
      const int al = tab.aT[k], ar = tab.aT[k + 1], bl = tab.bW[k], br = tab.bW[k + 1];
      mq::env_update(p, s, p.trial + tab.toff[k], al, ar, bl, br, W + tab.woff[k], bl, bl * br,
                     Fbuf + cur * fst, Fbuf + (1 - cur) * fst, (k > 0) ? tab.bondJ[k - 1] : 0.0, k == 0);
      cur = 1 - cur;
    }
    if (tid == 0) out[w] = Fbuf[cur * fst] / ov[w];
    __syncthreads();
  }
}

int err(int code, const std::string &m) {
  mq_host::set_last_error(m);
  return code;
}

bool dims_ok(const int *dims, int L) {
  if (dims[0] != 1 || dims[L] != 1) return false;
  for (int k = 0; k < L; ++k)
    if (dims[k] < 1 || dims[k + 1] < 1 || dims[k + 1] > 2 * dims[k] || dims[k] > 2 * dims[k + 1])
      return false;
  return true;
}

// One-time, per-device set-up with that device current.
int setup_device(int dev, DeviceSetup **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup &st = g_setup[dev];
  if (!st.ready) {
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess)
      return err(MPSQMC_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) return err(MPSQMC_E_CUDA, std::string("properties: ") + cudaGetErrorString(e));
    e = cudaFuncSetAttribute(energy_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)prop.sharedMemPerBlockOptin);
    if (e != cudaSuccess) return err(MPSQMC_E_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    st.scratch = static_cast<double *>(addr);
    st.sm_count = prop.multiProcessorCount;
    st.smem_optin = (int)prop.sharedMemPerBlockOptin;
    st.ready = true;
  }
  *out = &st;
  return 0;
}

}  // namespace

extern "C" int mpsqmc_local_energy_noalloc(const mpsqmc_energy_layout *lay, const double *trial,
                                           const double *walkers, long walker_stride,
                                           const double *overlaps, int n_walkers, double *energies,
                                           int device, void *stream) {
  if (!lay || !lay->trial_dims || !lay->walker_dims) return err(MPSQMC_E_ARG, "null layout");
  const int L = lay->L;
  if (lay->d != 2) return err(MPSQMC_E_UNSUPPORTED, "only d = 2 is implemented");
  if (L < 3 || L > kMaxL)
    return err(MPSQMC_E_UNSUPPORTED, "L outside [3, MPSQMC_NOALLOC_MAX_L = " + std::to_string(kMaxL) + "]");
  if (!dims_ok(lay->trial_dims, L) || !dims_ok(lay->walker_dims, L))
    return err(MPSQMC_E_ARG, "bond dimensions inconsistent with the chain");
  if (n_walkers < 0) return err(MPSQMC_E_ARG, "negative walker count");
  if (n_walkers > 0 && (!trial || !walkers || !overlaps || !energies))
    return err(MPSQMC_E_ARG, "null device pointer");
  if (lay->nC < 0 || (lay->nC > 0 && (!lay->ci || !lay->cj || !lay->cJ))) return err(MPSQMC_E_ARG, "bad couplings");
  Tables tab;
  std::memset(&tab, 0, sizeof tab);
  for (int c = 0; c < lay->nC; ++c) {
    const int i = lay->ci[c], j = lay->cj[c];
    if (i < 0 || j >= L || j != i + 1)
      return err(MPSQMC_E_UNSUPPORTED, "only nearest-neighbour chain couplings are implemented");
    tab.bondJ[i] += lay->cJ[c];
  }
  int maxA = 1, maxB = 1;
  long to = 0, wo = 0;
  for (int k = 0; k <= L; ++k) {
    tab.aT[k] = lay->trial_dims[k];
    tab.bW[k] = lay->walker_dims[k];
    maxA = std::max(maxA, tab.aT[k]);
    maxB = std::max(maxB, tab.bW[k]);
  }
  for (int k = 0; k < L; ++k) {
    tab.toff[k] = to;
    tab.woff[k] = wo;
    to += (long)tab.aT[k] * tab.aT[k + 1] * 2;
    wo += (long)tab.bW[k] * tab.bW[k + 1] * 2;
  }
  if (walker_stride < wo) return err(MPSQMC_E_ARG, "walker_stride smaller than one walker");
  // per CTA: the compact-MPO environments (2 x 4 blocks, ld maxA) and, when they do not fit in
  // shared memory beside the small buffers, the matrix work buffers (no Householder panel)
  const int pa = mq::padld(maxA), pb = mq::padld(maxB), pq = mq::padld(2 * maxB);
  long big_doubles = 0;
  double one = 0.0;
  const long smem_small = mq::smem_doubles(L, maxA, maxB, 1, pa, pb, pq, nullptr, nullptr, &one, &big_doubles,
                                           false, false);
  const long env_doubles = ((2L * 4 * maxA * maxB) + 31) & ~31L;
  const long avail = (long)kScratchDoubles;
  if (device < 0 || device >= kMaxDevices) return err(MPSQMC_E_ARG, "device ordinal out of range");
  if (env_doubles > avail)
    return err(MPSQMC_E_UNSUPPORTED, "bond dimensions need " + std::to_string(env_doubles * 8) +
                                         " bytes of scratch per CTA; the static array holds " +
                                         std::to_string(avail * 8));

  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return err(MPSQMC_E_NODEVICE, "no CUDA device");
  if (cudaSetDevice(device) != cudaSuccess) return err(MPSQMC_E_ARG, "cudaSetDevice failed");
  DeviceSetup *st = nullptr;
  int rc = setup_device(device, &st);
  if (rc == 0) {
    const bool on_chip = (smem_small + big_doubles) * (long)sizeof(double) <= (long)st->smem_optin;
    const long per_cta = on_chip ? env_doubles : env_doubles + ((big_doubles + 31) & ~31L);
    const size_t smem = sizeof(double) * (size_t)(on_chip ? smem_small + big_doubles : smem_small);
    if (per_cta > avail) {
      rc = err(MPSQMC_E_UNSUPPORTED, "bond dimensions need " + std::to_string(per_cta * 8) +
                                         " bytes of scratch per CTA; the static array holds " +
                                         std::to_string(avail * 8));
    } else if ((int)smem > st->smem_optin) {
      rc = err(MPSQMC_E_UNSUPPORTED, "bond dimensions exceed the shared-memory budget of one CTA");
    } else if (n_walkers > 0) {
      mq::Dev p;
      std::memset(&p, 0, sizeof p);
      p.L = L;
      p.d = 2;
      p.G = 1;
      p.maxA = maxA;
      p.maxB = maxB;
      p.pa = pa;
      p.pb = pb;
      p.pq = pq;
      p.trial = trial;
      p.h = lay->h;
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
          p.opSz[a + 2 * b] = (a == b) ? (a == 0 ? -0.5 : 0.5) : 0.0;
          p.opSx[a + 2 * b] = (a != b) ? 0.5 : 0.0;
          p.opISy[a + 2 * b] = (a == b + 1) ? 0.5 : ((a + 1 == b) ? -0.5 : 0.0);
        }
      p.scratch = st->scratch;
      p.scr_stride = per_cta;
      cudaStream_t s = static_cast<cudaStream_t>(stream);
      const int grid = (int)std::max(1L, std::min({(long)n_walkers, (long)st->sm_count, avail / per_cta}));
      energy_noalloc_kernel<<<grid, mq::kThreads, smem, s>>>(p, tab, on_chip ? -1L : env_doubles, walkers,
                                                           walker_stride, overlaps, energies, n_walkers);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) rc = err(MPSQMC_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    }
  }
  if (prev >= 0 && prev != device) cudaSetDevice(prev);
  return rc;
}
