// Host side of the tcgen05 products (tc_gemm.cuh): TMA tensor maps and launches, and the
// mpsqmc_tc_gemm entry point that exposes one batched product through the C ABI.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mpsqmc_gpu.h"
#include "tc_gemm.cuh"

namespace mq_host {
void set_last_error(const std::string &msg);  // capi.cu: backs mpsqmc_last_error()
}

namespace mq {
namespace tc {

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

int fail(int code, const std::string &m) {
  mq_host::set_last_error(m);
  return code;
}

}  // namespace

// A K-major FP32 operand as a 3D tensor map (k, row, z): element (k, r, z) at
// base[k + r * row_stride + z * z_stride]; box (kc, box_rows, box_z), 128-byte swizzle for kc = 32
// and 64-byte swizzle for kc = 16.
// k_ext, rows, zs: extents the loads may touch (allocated memory; padding must be zero where a
// product would read it).  Strides are in elements and must be multiples of 4 (16 bytes).
int make_operand_map(CUtensorMap *map, const float *base, long k_ext, long rows, long zs, long row_stride,
                     long z_stride, int box_rows, int box_z, int kc = kKC) {
  EncodeTiled enc = encoder();
  if (!enc) return fail(MPSQMC_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_stride & 3) || (z_stride & 3))
    return fail(MPSQMC_E_ARG, "tcgen05 operand: base and strides must be 16-byte aligned");
  if (box_rows < 1 || box_rows > 256 || box_z < 1 || box_z > 256)
    return fail(MPSQMC_E_ARG, "tcgen05 operand: box outside [1, 256]");
  cuuint64_t dims[3] = {(cuuint64_t)k_ext, (cuuint64_t)rows, (cuuint64_t)zs};
  cuuint64_t strides[2] = {(cuuint64_t)row_stride * 4, (cuuint64_t)std::max(z_stride, row_stride * rows) * 4};
  if (kc != 32 && kc != 16) return fail(MPSQMC_E_ARG, "tcgen05 operand: 16 or 32 k-values per stage");
  cuuint32_t box[3] = {(cuuint32_t)kc, (cuuint32_t)box_rows, (cuuint32_t)box_z};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, kc == 32 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MPSQMC_E_ARG, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return 0;
}

// Column-major D (element (m, n, z) at D[m + n dn + z dz]) as the epilogue's store map: box
// (box_rows, 16, 1), no swizzle; extents M x N x zs clip what a box holds past them.  Used when
// dn and dz are multiples of 4 and D is 16-byte aligned (else the epilogue stores directly).
bool make_store_map(CUtensorMap *map, float *D, long M, long N, long zs, long dn, long dz, int box_rows,
                    int box_cols = 16) {
  EncodeTiled enc = encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(D) & 15) || (dn & 3) || (dz & 3) || dn < M || (zs > 1 && dz < N * dn))
    return false;
  cuuint64_t dims[3] = {(cuuint64_t)M, (cuuint64_t)N, (cuuint64_t)std::max(1L, zs)};
  cuuint64_t strides[2] = {(cuuint64_t)dn * 4, (cuuint64_t)std::max(dz, N * dn) * 4};
  cuuint32_t box[3] = {(cuuint32_t)box_rows, (cuuint32_t)box_cols, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, D, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// Row-major D (element (m, n, z) at D[n + m dm + z dz]) as the epilogue's store map: box
// (32, box_rows, 1) with a 128-byte swizzle; extents N x M x zs clip what a box holds past them.
bool make_row_store_map(CUtensorMap *map, float *D, long M, long N, long zs, long dm, long dz, int box_rows) {
  EncodeTiled enc = encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(D) & 15) || (dm & 3) || (dz & 3) || dm < N || (zs > 1 && dz < M * dm))
    return false;
  cuuint64_t dims[3] = {(cuuint64_t)N, (cuuint64_t)M, (cuuint64_t)std::max(1L, zs)};
  cuuint64_t strides[2] = {(cuuint64_t)dm * 4, (cuuint64_t)std::max(dz, M * dm) * 4};
  cuuint32_t box[3] = {32, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, D, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// The epilogue's store route: TMA boxes for column-major outputs without accumulation, 32 columns
// wide for unstacked tiles whose width is a multiple of 32 (dsplit, set later, narrows them), and
// for row-major ones whose 32-column steps stay in one batch entry.
void pick_store(GemmParams &p, long zs) {
  p.dtma = p.dwide = p.rtma = 0;
  if (p.epi == kStore && p.dn == 1 && p.dm > 1 && !p.beta && (p.tn & 31) == 0 &&
      (p.bstack == 1 || (p.N & 31) == 0)) {
    p.rtma = make_row_store_map(&p.tmD, p.D, p.M, p.N, zs, p.dm, p.dz, p.tm == 128 ? 32 : 16) ? 1 : 0;
    return;
  }
  if (p.epi == kStore && p.dm == 1 && !p.beta && p.dn > 1) {
    const int wide = p.bstack == 1 && (p.tn & 31) == 0;
    p.dtma = make_store_map(&p.tmD, p.D, p.M, p.N, zs, p.dn, p.dz, p.tm == 128 ? 32 : 16, wide ? 32 : 16) ? 1 : 0;
    p.dwide = p.dtma && wide;
  }
}

// SM count and the dynamic shared memory a launch may use (the opt-in limit less the kernel's
// static barriers), set once per process.
int configure_kernel(int *sms, int *smem_limit) {
  static int n_sms = 0, limit = 0;
  static std::once_flag once;
  static cudaError_t status = cudaSuccess;
  std::call_once(once, [] {
    int dev = 0, optin = 0;
    status = cudaGetDevice(&dev);
    if (status == cudaSuccess) status = cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev);
    if (status == cudaSuccess) status = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    limit = optin - 2048;
    if (status == cudaSuccess)
      status = cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
  });
  if (status != cudaSuccess) return fail(MPSQMC_E_CUDA, std::string("tcgen05 GEMM set-up: ") + cudaGetErrorString(status));
  *sms = n_sms;
  if (smem_limit) *smem_limit = limit;
  return 0;
}

// The load ring's depth for this tile shape (as deep as shared memory allows, at most max_stages).
int pick_stages(GemmParams &p, int max_stages = kMaxStages) {
  int sms = 0, limit = 0;
  const int rc = configure_kernel(&sms, &limit);
  if (rc) return rc;
  p.stages = std::max(2, std::min(max_stages, stages_for(p.tm, p.tn, p.passes, limit, p.dsplit, p.kc, p.bf16)));
  if (smem_bytes(p.tm, p.tn, p.passes, p.stages, p.dsplit, p.kc, p.bf16) > limit)
    return fail(MPSQMC_E_UNSUPPORTED, "tcgen05 GEMM tile does not fit in shared memory");
  return 0;
}

// Launch one batched product; max_tiles bounds the grid (the persistent CTAs loop over tiles).
int launch(const GemmParams &p, long max_tiles, cudaStream_t stream) {
  int sms = 0;
  int rc = configure_kernel(&sms, nullptr);
  if (rc) return rc;
  const int grid = (int)std::max(1L, std::min((long)sms, max_tiles));
  tc_gemm_kernel<<<grid, kThreads, smem_bytes(p.tm, p.tn, p.passes, p.stages, p.dsplit, p.kc, p.bf16), stream>>>(p);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MPSQMC_E_CUDA, std::string("tcgen05 GEMM launch: ") + cudaGetErrorString(e));
  return 0;
}

}  // namespace tc
}  // namespace mq

extern "C" int mpsqmc_tc_gemm(float *D, const float *A, const float *B, int M, int N, int K, long lda,
                              long a_zstride, int adiv, long a_zcount, long ldb, long b_zstride, int bdiv,
                              long b_zcount, int Z, int bstack, float alpha, int beta, int passes, long dz,
                              long dm, long dn, int *err, void *stream) {
  using namespace mq::tc;
  if (!D || !A || !B || !err) return fail(MPSQMC_E_ARG, "null pointer");
  if (M < 1 || N < 1 || K < 1 || Z < 1 || bstack < 1) return fail(MPSQMC_E_ARG, "sizes must be positive");
  if (passes != 1 && passes != 3 && passes != kPassesBF16)
    return fail(MPSQMC_E_ARG, "passes must be 1, 3 or 16 (one BF16 pass)");
  if (lda < ((K + kKC - 1) / kKC) * kKC || ldb < ((K + kKC - 1) / kKC) * kKC)
    return fail(MPSQMC_E_ARG, "lda and ldb must cover K rounded up to a multiple of 32 (zero padded)");
  GemmParams p;
  std::memset(&p, 0, sizeof p);
  p.M = M;
  p.N = N;
  p.K = K;
  p.tm = M <= 64 ? 64 : 128;
  if (bstack > 1) {
    if (adiv != 0) return fail(MPSQMC_E_ARG, "stacking batch entries along N needs a shared A (adiv = 0)");
    if ((N & 7) || N * bstack > kMaxTN) return fail(MPSQMC_E_ARG, "stacked tile: N multiple of 8, N * bstack <= 256");
    p.tn = (N * bstack + 15) & ~15;
    p.brows = N;
  } else {
    p.tn = std::min(kMaxTN, (N + 15) & ~15);
    p.brows = p.tn;
  }
  p.adiv = adiv;
  p.bdiv = bdiv;
  p.bstack = bstack;
  p.Z = Z;
  p.alpha = alpha;
  p.beta = beta;
  p.passes = passes == kPassesBF16 ? 1 : passes;
  p.bf16 = passes == kPassesBF16;
  p.D = D;
  p.dz = dz;
  p.dm = dm;
  p.dn = dn;
  p.epi = kStore;
  p.err = err;
  p.kc = kKC;
  const long kpad = ((K + kKC - 1) / kKC) * kKC;
  // operand rows the boxes may touch: whole tiles (callers pad A to a multiple of tm rows and
  // B to a multiple of the tile rows when bstack == 1)
  const long arows = ((M + p.tm - 1) / p.tm) * p.tm;
  const long brows = bstack > 1 ? N : ((N + p.tn - 1) / p.tn) * p.tn;
  int rc = pick_stages(p);
  pick_store(p, Z);
  if (!rc) rc = make_operand_map(&p.tmA, A, kpad, arows, std::max(1L, a_zcount), lda, a_zstride, p.tm, 1, p.kc);
  if (!rc) rc = make_operand_map(&p.tmB, B, kpad, brows, std::max(1L, b_zcount), ldb, b_zstride, p.brows, bstack, p.kc);
  if (rc) return rc;
  const long mt = (M + p.tm - 1) / p.tm;
  const long nt = bstack > 1 ? (Z + bstack - 1) / bstack : (long)Z * ((N + p.tn - 1) / p.tn);
  return launch(p, mt * nt, static_cast<cudaStream_t>(stream));
}

// =============================================================================================
// The walker-batched sweep (batched.h)
// =============================================================================================
#include <functional>
#include <vector>

#include "batched.h"

namespace mq {
namespace bs {

using namespace mq::tc;

namespace {

constexpr int kTraceStride = 21;
constexpr int kErrNumeric = 1, kErrCapacity = 2;

inline long pad4(long x) { return (x + 3) & ~3L; }
inline long pad64(long x) { return (x + 63) & ~63L; }
inline int tm_for(int M) { return M <= 64 ? 64 : 128; }

// x rounded to the nearest TF32 value, ties away from zero (the device's cvt.rna.tf32.f32): the
// 13 low mantissa bits are rounded off the magnitude
inline float tf32_round(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;
  u = (u + 0x1000u) & ~0x1fffu;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// ---------------------------------------------------------------------------------------------
// Small kernels (FP64 bookkeeping and elementwise steps).  w: logical walker index; every kernel
// covers w < min(*n_cur, cap).
// ---------------------------------------------------------------------------------------------
struct SiteForms {          // device tables, one entry per site
  const long *woff;         // FP64 offset of site k in a walker slot
  const int *bl, *br;       // walker bond dims of site k
  const long *sl_off, *sr_off;  // site k's FP32 forms inside the SL / SR arrays
  const long *sl_sz, *sr_sz;    // floats per walker of site k's forms
  const long *sl_ld, *sr_ld;    // their row strides
};

// FP64 walker sites -> the two FP32 forms: SL_k[(2c + s) ldl + r] (rows (c, sigma), k = the left
// bond) and SR_k[(2r + s) ldr + c] (rows (r, sigma), k = the right bond).  Interleaving sigma in the
// rows lets the sums over sigma of the trial products run as one product with sigma stacked along K.
// One element of a site form from the FP64 walker: its FP32 value, or (tail != 0, three passes)
// its TF32 head at p[i] and the TF32 rounding of what the head misses at p[tail + i].
__device__ __forceinline__ void put_form(float *p, long tail, long i, double y) {
  if (!tail) {
    p[i] = (float)y;
    return;
  }
  const float h = to_tf32((float)y);
  p[i] = h;
  p[tail + i] = to_tf32((float)(y - (double)h));
}

__global__ void convert_kernel(SiteForms f, const double *walkers, long wstride, const int *slot_of, const int *n_cur,
                               int cap, float *SL, float *SR, long slt, long srt) {
  const int k = blockIdx.y;
  const int N = min(*n_cur, cap);
  const int bl = f.bl[k], br = f.br[k];
  const long per = 2L * bl * br;
  const long ldl = f.sl_ld[k], ldr = f.sr_ld[k];
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < per * N; e += (long)gridDim.x * blockDim.x) {
    const int w = (int)(e / per);
    const long q = e % per;
    const int r = (int)(q % bl), c = (int)((q / bl) % br), s = (int)(q / ((long)bl * br));
    const double x = walkers[(long)slot_of[w] * wstride + f.woff[k] + q];
    put_form(SL, slt, f.sl_off[k] + (long)w * f.sl_sz[k] + (2L * c + s) * ldl + r, x);
    put_form(SR, srt, f.sr_off[k] + (long)w * f.sr_sz[k] + (2L * r + s) * ldr + c, x);
  }
}

// Per walker: weight copy, unit left environments at site 0, R_L = 1.
// nb: the walkers this step's products cover, min(n_cur, cap).
__global__ void init_kernel(const double *weight, const int *slot_of, const int *n_cur, int cap, double *wtb,
                            float *Lenv, long lsz, float *Nl, long nsz, float *RL, long rsz, int *err, int *nb) {
  const int N = *n_cur;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (N > cap) atomicOr(err, kErrCapacity);
    *nb = min(N, cap);
  }
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < min(N, cap); w += gridDim.x * blockDim.x) {
    wtb[w] = weight[slot_of[w]];
    Lenv[(long)w * lsz] = 1.f;
    Nl[(long)w * nsz] = 1.f;
    RL[(long)w * rsz] = 1.f;
  }
}

// ov = sum_s B_0[s](0, a) R_1(a, b) A_0[s](0, b) (site 0 has left bond 1).  One warp per walker.
__global__ void overlap0_kernel(const double *trial, int a1, int b1, const float *R1, long r1sz, long r1ld,
                                const double *walkers, long wstride, const int *slot_of, const int *n_cur, int cap,
                                double *ovb) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= min(*n_cur, cap)) return;
  const double *W = walkers + (long)slot_of[w] * wstride;
  double part = 0.0;
  for (int q = lane; q < 2 * a1 * b1; q += 32) {
    const int a = q % a1, b = (q / a1) % b1, s = q / (a1 * b1);
    part += trial[a + a1 * s] * (double)R1[(long)w * r1sz + a * r1ld + b] * W[b + b1 * s];
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) ovb[w] = part;
}

// C_kl from the closures, PDF, weight, CDF sample and the site operators of coupling c (the
// arithmetic of MPSQMC2.cpp:540-588 and MPSstate.cpp:575-633 as walker_general.cuh's
// sample_coupling does it).  One warp per walker; 4 warps per block.
__global__ void __launch_bounds__(128) sample_kernel(const double *dot, const double *U, const double *Sq,
                                                     const double *VT, const double *grid, int G, const double *uni,
                                                     int nC, int c, const int *n_cur, int cap, double *ovb,
                                                     double *wtb, double *ob, double *trace) {
  __shared__ double pdf_s[4][256];
  __shared__ double cm_s[4][16];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int w = blockIdx.x * 4 + wl;
  if (w >= min(*n_cur, cap)) return;
  const double *M = dot + (long)w * 16;
  if (lane < 16) {
    const int k = lane & 3, l = lane >> 2;
    double acc = 0.0;
    for (int qq = 0; qq < 4; ++qq) {
      double inner = 0.0;
      for (int pp = 0; pp < 4; ++pp) inner += U[pp + 4 * k] * M[pp + 4 * qq];
      acc += inner * VT[l + 4 * qq];
    }
    cm_s[wl][k + 4 * l] = Sq[k] * Sq[l] * acc;
  }
  __syncwarp();
  const double *Cm = cm_s[wl];
  const double ov = ovb[w];
  const double fac = 4.0 / (ov * G);
  double part = 0.0;
  for (int g = lane; g < G; g += 32) {
    const double *x = grid + 4 * g;
    double v = 0.0;
    for (int l = 0; l < 4; ++l)
      for (int r = 0; r < 4; ++r) v += Cm[l + 4 * r] * x[l] * x[r];
    v = fmax(0.0, v) * fac;
    pdf_s[wl][g] = v;
    part += v;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  const double pnorm = part;
  const double pinv = 1.0 / pnorm;
  for (int g = lane; g < G; g += 32) pdf_s[wl][g] *= pinv;
  __syncwarp();
  if (lane == 0) {
    const double u = uni[(long)w * nC + c];
    int count = 0;
    double cum = pdf_s[wl][0];
    while ((cum <= u) && (count < G - 1)) {
      count += 1;
      cum += pdf_s[wl][count];
    }
    const double *x = grid + 4 * count;
    double nm = 0.0;
    for (int l = 0; l < 4; ++l)
      for (int r = 0; r < 4; ++r) nm += Cm[l + 4 * r] * x[l] * x[r];
    const double wt = wtb[w] * pnorm;
    wtb[w] = wt;
    ovb[w] = 4.0 * nm;
    for (int q = 0; q < 4; ++q) {
      double o1 = 0.0, o2 = 0.0;
      for (int k = 0; k < 4; ++k) {
        const double pf = 2.0 * Sq[k] * x[k];
        o1 += pf * U[q + 4 * k];
        o2 += pf * VT[k + 4 * q];
      }
      ob[(long)w * 8 + q] = o1;
      ob[(long)w * 8 + 4 + q] = o2;
    }
    if (trace) {
      double *t = trace + ((long)w * nC + c) * kTraceStride;
      for (int k = 0; k < 16; ++k) t[k] = Cm[k] / ov;
      t[16] = pnorm;
      t[17] = u;
      t[18] = count;
      t[19] = wt;
      t[20] = 4.0 * nm / ov;
    }
  }
}

// O1 (ob[0..3]) on site i and O2 (ob[4..7]) on site j of every walker: the FP64 slot and both FP32
// forms.  blockIdx.y = 0: site i, 1: site j.
__global__ void site_op_kernel(SiteForms f, int si, int sj, const double *ob, double *walkers, long wstride,
                               const int *slot_of, const int *n_cur, int cap, float *SL, float *SR, long slt,
                               long srt) {
  const int k = blockIdx.y == 0 ? si : sj;
  const int oo = blockIdx.y == 0 ? 0 : 4;
  const int N = min(*n_cur, cap);
  const int bl = f.bl[k], br = f.br[k];
  const long blk = (long)bl * br;
  const long ldl = f.sl_ld[k], ldr = f.sr_ld[k];
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < blk * N; e += (long)gridDim.x * blockDim.x) {
    const int w = (int)(e / blk);
    const long q = e % blk;
    const int r = (int)(q % bl), c = (int)(q / bl);
    const double *O = ob + (long)w * 8 + oo;
    double *X = walkers + (long)slot_of[w] * wstride + f.woff[k];
    const double x0 = X[q], x1 = X[blk + q];
    const double y0 = O[0] * x0 + O[2] * x1, y1 = O[1] * x0 + O[3] * x1;
    X[q] = y0;
    X[blk + q] = y1;
    float *sl = SL + f.sl_off[k] + (long)w * f.sl_sz[k];
    float *sr = SR + f.sr_off[k] + (long)w * f.sr_sz[k];
    put_form(sl, slt, 2L * c * ldl + r, y0);
    put_form(sl, slt, (2L * c + 1) * ldl + r, y1);
    put_form(sr, srt, 2L * r * ldr + c, y0);
    put_form(sr, srt, (2L * r + 1) * ldr + c, y1);
  }
}

// QR-free sweep: the finished centre (site i) rescaled to the Frobenius norm of an isometry,
// sqrt(b_r); the overlap takes the same factor (walker_general.cuh).  One block per walker.
__global__ void rescale_kernel(SiteForms f, int k, double *walkers, long wstride, const int *slot_of, const int *n_cur,
                               int cap, float *SL, float *SR, long slt, long srt, double *ovb, double *scl) {
  __shared__ double red[8];
  const int w = blockIdx.x;
  if (w >= min(*n_cur, cap)) return;
  const int bl = f.bl[k], br = f.br[k];
  const long n = 2L * bl * br;
  double *X = walkers + (long)slot_of[w] * wstride + f.woff[k];
  double part = 0.0;
  for (long q = threadIdx.x; q < n; q += blockDim.x) part += X[q] * X[q];
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  double tot = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot += red[i];
  const double inv = sqrt((double)br / tot);
  const long ldl = f.sl_ld[k], ldr = f.sr_ld[k];
  float *sl = SL + f.sl_off[k] + (long)w * f.sl_sz[k];
  float *sr = SR + f.sr_off[k] + (long)w * f.sr_sz[k];
  for (long q = threadIdx.x; q < n; q += blockDim.x) {
    const double y = X[q] * inv;
    X[q] = y;
    const int r = (int)(q % bl), c = (int)((q / bl) % br), s = (int)(q / ((long)bl * br));
    put_form(sl, slt, (2L * c + s) * ldl + r, y);
    put_form(sr, srt, (2L * r + s) * ldr + c, y);
  }
  if (threadIdx.x == 0) {
    ovb[w] *= inv;
    scl[w] = inv;
  }
}

// The final site's left branches from the last coupling's (P is linear in the centre's sigma
// blocks): P'[s, t] = inv sum_t' O1(t, t') P[s, t'].
__global__ void derive_p_kernel(float *P, long psz, long pld, int a, int b, const double *ob, const double *scl,
                                const int *n_cur, int cap) {
  const int N = min(*n_cur, cap);
  const long blk = (long)a * b;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < blk * N; e += (long)gridDim.x * blockDim.x) {
    const int w = (int)(e / blk);
    const long q = e % blk;
    const long off = (q / b) * pld + q % b;
    const double inv = scl[w];
    const double *O = ob + (long)w * 8;
    const float o0 = (float)(inv * O[0]), o1 = (float)(inv * O[1]), o2 = (float)(inv * O[2]),
                o3 = (float)(inv * O[3]);
    float *Pw = P + (long)w * 4 * psz;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      float *P0 = Pw + (long)s * psz + off, *P1 = Pw + (long)(s + 2) * psz + off;
      const float x0 = *P0, x1 = *P1;
      *P0 = o0 * x0 + o2 * x1;
      *P1 = o1 * x0 + o3 * x1;
    }
  }
}

struct EnvOps {
  double opSx[4], opISy[4], opSz[4];
};

// done' (+)= -h sum_e Sz[e] P_e (the field closes on the site) over a_{k+1} x b_{k+1}; add: the
// products of the closing channels are already in Fdn.
__global__ void env_init_kernel(const float *P, long psz, long pld, int a, int b, float *Fdn, long fsz, long fld,
                                double h, EnvOps ops, int add, const int *n_cur, int cap) {
  const int N = min(*n_cur, cap);
  const long blk = (long)a * b;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < blk * N; e += (long)gridDim.x * blockDim.x) {
    const int w = (int)(e / blk);
    const long q = e % blk;
    const long r = q / b, c = q % b;
    const float *Pw = P + (long)w * 4 * psz + r * pld + c;
    float fz = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) fz += (float)ops.opSz[k] * Pw[k * psz];
    float *f = Fdn + (long)w * fsz + r * fld + c;
    *f = add ? *f + (float)(-h) * fz : (float)(-h) * fz;
  }
}

// G[t](r, c) = delta_st Fd + sum_e J_e (Sx(s,t) F_x - iSy(s,t) F_y + Sz(s,t) F_z) for the channels
// e closing on site k (a_k x b_k), sigma = s; stored Gb[r (2 gld) + t gld + c] (t stacked along K).
__global__ void gbuild_kernel(const float *Fd, long fsz, long fld, const float *Fch, long csz, int nslots,
                              const int *eslot, const float *eJ, int ne, int a, int b, EnvOps ops, float *Gb,
                              long gsz, long gsig, long gld, const int *n_cur, int cap) {
  // both sigma blocks of the site's operator rows from one read of Fd and the closing channels:
  // G_s[t] = delta_st Fd + sum_e J_e (op_x[s + 2t] F_x - op_iy[s + 2t] F_iy + op_z[s + 2t] F_z)
  const int N = min(*n_cur, cap);
  const long blk = (long)a * b;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < blk * N; e += (long)gridDim.x * blockDim.x) {
    const int w = (int)(e / blk);
    const long q = e % blk;
    const long off = (q / b) * fld + q % b;
    const float fd = Fd[(long)w * fsz + off];
    float gx = 0.f, gy = 0.f, gz = 0.f;
    for (int i = 0; i < ne; ++i) {
      const float *F = Fch + ((long)w * nslots * 3 + 3L * eslot[i]) * csz + off;
      gx += eJ[i] * F[0];
      gy += eJ[i] * F[csz];
      gz += eJ[i] * F[2 * csz];
    }
    float *Gw = Gb + (long)w * gsz + (q / b) * 2 * gld + q % b;
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int o = s + 2 * t;
        Gw[s * gsig + t * gld] =
            ((s == t) ? fd : 0.f) + (float)ops.opSx[o] * gx - (float)ops.opISy[o] * gy + (float)ops.opSz[o] * gz;
      }
  }
}

// Lenv' = P[0,0] + P[1,1]; the channel site k opens (slot >= 0): F[a] = sum_e op_a[e] P_e.
__global__ void env_finish_kernel(const float *P, long psz, long pld, int a, int b, float *Lenv, long lsz, float *Fch,
                                  long csz, int nslots, int slot, EnvOps ops, const int *n_cur, int cap) {
  const int N = min(*n_cur, cap);
  const long blk = (long)a * b;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < blk * N; e += (long)gridDim.x * blockDim.x) {
    const int w = (int)(e / blk);
    const long q = e % blk;
    const long off = (q / b) * pld + q % b;
    const float *Pw = P + (long)w * 4 * psz + off;
    float p[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) p[k] = Pw[k * psz];
    Lenv[(long)w * lsz + off] = p[0] + p[3];
    if (slot >= 0) {
      float fx = 0.f, fy = 0.f, fz = 0.f;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        fx += (float)ops.opSx[k] * p[k];
        fy += (float)ops.opISy[k] * p[k];
        fz += (float)ops.opSz[k] * p[k];
      }
      float *F = Fch + ((long)w * nslots * 3 + 3L * slot) * csz + off;
      F[0] = fx;
      F[csz] = fy;
      F[2 * csz] = fz;
    }
  }
}

// Last site: energy and overlap of the unnormalised walker, its norm through the left norm
// environment, normalisation of the FP64 site L-1 and the per-walker outputs.  One warp per walker.
__global__ void final_kernel(int bl, long woff, double *walkers, long wstride, const int *slot_of, const float *Nl,
                             long nsz, long nld, const float *Lenv, long lsz, const float *Fdn, long fsz,
                             const double *wtb, double *overlap, double *weight, double *energy, double *ov_out,
                             double *wt_out, const int *n_cur, int cap, int *err) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= min(*n_cur, cap)) return;
  const int slot = slot_of[w];
  double *X = walkers + (long)slot * wstride + woff;  // site L-1: bl x 1 per sigma
  double part = 0.0;
  for (int q = lane; q < 2 * bl; q += 32) {
    const int r = q % bl, s = q / bl;
    double y = 0.0;
    for (int k = 0; k < bl; ++k) y += (double)Nl[(long)w * nsz + (long)r * nld + k] * X[s * bl + k];
    part += X[q] * y;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  const double nrm = sqrt(part);
  const double ovr = Lenv[(long)w * lsz], en = Fdn[(long)w * fsz];
  const double scale = (ovr < 0.0) ? -1.0 / nrm : 1.0 / nrm;
  __syncwarp();
  for (int q = lane; q < 2 * bl; q += 32) X[q] *= scale;
  if (lane == 0) {
    const double ovf = fabs(ovr) / nrm, ew = en / ovr, wt = wtb[w];
    overlap[slot] = ovf;
    weight[slot] = wt;
    energy[w] = ew;
    ov_out[w] = ovf;
    wt_out[w] = wt;
    if (!(isfinite(wt) && isfinite(ovf) && isfinite(ew))) atomicOr(err, kErrNumeric);
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// The plan
// ---------------------------------------------------------------------------------------------
struct Plan {
  Problem pr;
  int cap = 0, sms = 1;
  std::vector<void *> allocs;
  size_t bytes = 0;
  // FP32 trial copies: TO_k[s] rows c < a_{k+1}, k = r (ld pad4(a_k)); TT_k[s] rows r < a_k, k = c
  std::vector<long> to_off, tt_off;  // per (k, s): k * 2 + s
  float *TO = nullptr, *TT = nullptr;
  // the same with sigma stacked along K in blocks of the contracted bond padded to 4 (so that K =
  // 2 pad4(bond) at every site, not twice the largest bond): TOs_k[c][s l + r] = B_k[s](r, c)
  // with l = pad4(a_k), TTs_k[r][s l' + c] = B_k[s](r, c) with l' = pad4(a_{k+1}); zero beyond
  // the site's bond
  std::vector<long> tos_off, tts_off;  // per k
  float *TOs = nullptr, *TTs = nullptr;
  // walker forms and right environments
  std::vector<long> sl_off, sr_off, sl_sz, sr_sz, sl_ld, sr_ld, r_off, r_sz, r_ld;
  float *SL = nullptr, *SR = nullptr, *R = nullptr;
  long slt = 0, srt = 0;           // three passes: offset of the site forms' TF32 tails (0: FP32 values)
  // work buffers (per walker, fixed strides)
  long ldA = 0, ldB = 0;           // pad4(maxA), pad4(maxB)
  long szBl = 0;                   // maxA x ldB (a row-major a x b block)
  long szX = 0;                    // 2 maxB x ldA (a column-major block with sigma-stacked rows)
  long szN = 0;                    // maxB x ldB
  long szW = 0;                    // 2 maxB x ldB
  float *Fdn_ptr(int fd) { return Fd[1 - fd]; }
  float *Lenv = nullptr, *P = nullptr, *X = nullptr, *X4 = nullptr, *Y = nullptr, *Nl[2] = {nullptr, nullptr},
        *Wn = nullptr, *Fd[2] = {nullptr, nullptr}, *Gb = nullptr, *Q = nullptr, *Fch = nullptr, *Xch = nullptr;
  // three passes: the trial copies hold [values | TF32 heads | TF32 tails] (sections of nto,
  // ntt, ntos, ntts floats), and the right factors of the trial products (X, X4, Y, Q, Xch) are
  // written as heads, with their tails in these arrays
  long nto = 0, ntt = 0, ntos = 0, ntts = 0;
  float *Xl = nullptr, *X4l = nullptr, *Yl = nullptr, *Ql = nullptr, *Xchl = nullptr;
  double *ovb = nullptr, *wtb = nullptr, *scl = nullptr, *ob = nullptr, *dot = nullptr;
  int *nb = nullptr;               // min(n_cur, cap), written at the step start: the products' walker count
  SiteForms sf;
  int *ech_slot_d = nullptr;
  float *ech_J_d = nullptr;
  int *err_tc = nullptr;
  std::vector<std::function<int(cudaStream_t, double *)>> ops;
  int launches = 0;
};

namespace {

template <typename T>
int palloc(Plan *p, T **ptr, size_t n) {
  const size_t b = std::max<size_t>(n, 1) * sizeof(T);
  void *v = nullptr;
  if (cudaMalloc(&v, b) != cudaSuccess) {
    cudaGetLastError();
    return fail(MPSQMC_E_CUDA, "batched sweep: device allocation of " + std::to_string(b) + " bytes failed");
  }
  if (cudaMemset(v, 0, b) != cudaSuccess) return fail(MPSQMC_E_CUDA, "batched sweep: memset failed");
  p->allocs.push_back(v);
  p->bytes += b;
  *ptr = static_cast<T *>(v);
  return 0;
}

// A K-major operand: element (k, row, z) at base[k + row ld + z zs].
struct Opnd {
  const float *base;
  long ld, rows, zs, zn;  // row stride, rows, z stride, z count (allocated)
  int div;                // z -> operand index divisor (0: shared)
  const float *hi = nullptr, *lo = nullptr;  // the same operand as TF32 head and tail arrays
};

// One batched product over zper * n_cur batch entries (per walker: zper consecutive entries).
// With three passes, operands that carry head and tail arrays are loaded split (both must), and
// Dlo asks for D as head (D) and tail (Dlo) arrays.
int add_gemm(Plan *p, const Opnd &A, const Opnd &B, int M, int N, int K, int zper, float *D, long dz, long dm, long dn,
             int beta, float alpha = 1.f, const float *E = nullptr, long ez = 0, long eq = 0, long em = 0, long en = 0,
             int doff = 0, float *Dlo = nullptr) {
  if (M < 1 || N < 1 || K < 1) return 0;
  GemmParams g;
  std::memset(&g, 0, sizeof g);
  g.M = M;
  g.N = N;
  g.K = K;
  g.tm = tm_for(M);
  const Tiles &t = p->pr.tiles;
  g.bf16 = p->pr.bf16 ? 1 : 0;
  // k-values per stage (the trial products' is a tile choice; BF16 stages take 32)
  g.kc = (A.div == 0 && !g.bf16) ? t.kc_trial : kKC;
  int bstack = 1;
  if (A.div == 0 && (N & 7) == 0 && 2 * N <= t.stack_tn) bstack = t.stack_tn / N;
  if (bstack > 1) {
    g.tn = (N * bstack + 15) & ~15;  // the MMA's N: a multiple of 16 (columns past N bstack unused)
    g.brows = N;
  } else {
    g.tn = std::min(A.div == 0 ? t.stack_tn : t.wide_tn, (N + 15) & ~15);
    g.brows = g.tn;
  }
  g.bstack = bstack;
  g.adiv = A.div;
  g.bdiv = B.div;
  g.Z = zper;
  g.zcount = p->nb;
  g.alpha = alpha;
  g.beta = beta;
  g.passes = p->pr.passes;
  g.D = D;
  g.dz = dz;
  g.dm = dm;
  g.dn = dn;
  g.err = p->pr.err;  // a pipeline wait that timed out sets kErrTimeout in the engine's error word
  if (E) {
    g.epi = kDot4;
    g.E = E;
    g.ez = ez;
    g.eq = eq;
    g.em = em;
    g.en = en;
    g.dot = p->dot;
    g.dstride = 16;
    g.doff = doff;
  }
  pick_store(g, (long)zper * p->cap);
  const bool three = p->pr.passes == 3;
  if (three && Dlo) {
    // the consumer loads this output split: only the TMA store route writes the two arrays
    if (!g.dtma || !make_store_map(&g.tmD2, Dlo, M, N, (long)zper * p->cap, dn, dz, g.tm == 128 ? 32 : 16) ||
        !make_store_map(&g.tmD, D, M, N, (long)zper * p->cap, dn, dz, g.tm == 128 ? 32 : 16))
      return fail(MPSQMC_E_UNSUPPORTED, "batched sweep: a split output needs the TMA store route");
    g.dsplit = 1;
    g.dwide = 0;  // head and tail boxes of 16 columns
  }
  g.presplit = three ? ((A.lo ? 1 : 0) | (B.lo ? 2 : 0)) : 0;
  const float *ah = (g.presplit & 1) ? A.hi : A.base, *bh = (g.presplit & 2) ? B.hi : B.base;
  const long brows_map = bstack > 1 ? N : B.rows;
  int rc = pick_stages(g, t.max_stages);
  if (!rc) rc = make_operand_map(&g.tmA, ah, K, A.rows, std::max(1L, A.zn), A.ld, A.zs, g.tm, 1, g.kc);
  if (!rc) rc = make_operand_map(&g.tmB, bh, K, brows_map, std::max(1L, B.zn), B.ld, B.zs, g.brows, bstack, g.kc);
  if (!rc && (g.presplit & 1))
    rc = make_operand_map(&g.tmA2, A.lo, K, A.rows, std::max(1L, A.zn), A.ld, A.zs, g.tm, 1, g.kc);
  if (!rc && (g.presplit & 2))
    rc = make_operand_map(&g.tmB2, B.lo, K, brows_map, std::max(1L, B.zn), B.ld, B.zs, g.brows, bstack, g.kc);
  if (rc) return rc;
  const long zt = (long)zper * p->cap;
  const long mt = (M + g.tm - 1) / g.tm;
  const long nt = bstack > 1 ? (zt + bstack - 1) / bstack : zt * ((N + g.tn - 1) / g.tn);
  const long tiles = mt * nt;
  p->ops.push_back([g, tiles](cudaStream_t s, double *) { return launch(g, tiles, s); });
  p->launches += 1;
  return 0;
}

int grid_elems(const Plan *p, long per_walker) {
  const long n = per_walker * p->cap;
  return (int)std::max(1L, std::min((n + 255) / 256, 8L * p->sms));
}

}  // namespace

size_t bytes_needed(const Problem &pr) {
  const int L = pr.L;
  const long maxA = *std::max_element(pr.aT.begin(), pr.aT.end()), maxB = *std::max_element(pr.bW.begin(), pr.bW.end());
  const long ldA = pad4(maxA), ldB = pad4(maxB);
  long per = 0;  // floats per walker
  const int forms = pr.passes == 3 ? 2 : 1;  // site forms as TF32 heads and tails with three passes
  for (int k = 0; k < L; ++k) {
    per += forms * (pad64(2L * pr.bW[k + 1] * pad4(pr.bW[k])) + pad64(2L * pr.bW[k] * pad4(pr.bW[k + 1])));
    per += pad64((long)pr.aT[k + 1] * pad4(pr.bW[k + 1]));
  }
  const long szBl = pad64(maxA * ldB), szX = pad64(2 * maxB * ldA), szN = pad64(maxB * ldB), szW = pad64(2 * maxB * ldB);
  const int ns = std::max(1, pr.nslots);
  per += szBl * (1 + 4 + 2 + 4 + 3L * ns) + szX * (1 + 4 + 1 + 3L * ns) + 2 * szN + szW + pad64(2 * maxB * ldA);
  if (pr.passes == 3) {  // tails of the right factors stored split
    const int sb = pr.tiles.split_out;
    per += szX * (((sb & kSplitY) ? 1 : 0) + ((sb & kSplitX) ? 1 : 0) + ((sb & kSplitX4) ? 4 : 0) +
                  ((sb & kSplitXch) ? 3L * ns : 0)) +
           ((sb & kSplitQ) ? pad64(2 * maxB * ldA) : 0);
  }
  return (size_t)per * pr.capacity * sizeof(float) + (size_t)pr.capacity * 48 * sizeof(double);
}

int build(const Problem &pr, Plan **out) {
  *out = nullptr;
  Plan *p = new Plan();
  p->pr = pr;
  auto bail = [&](int rc) {
    destroy(p);
    return rc;
  };
  const int L = pr.L;
  const std::vector<int> &a = pr.aT, &b = pr.bW;
  p->cap = pr.capacity;
  if (pr.G > 256) return bail(fail(MPSQMC_E_UNSUPPORTED, "the tcgen05 sweep samples grids of at most 256 points"));
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return bail(fail(MPSQMC_E_CUDA, "batched sweep: device query failed"));
  const long maxA = *std::max_element(a.begin(), a.end()), maxB = *std::max_element(b.begin(), b.end());
  p->ldA = pad4(maxA);
  p->ldB = pad4(maxB);
  p->szBl = pad64(maxA * p->ldB);
  p->szX = pad64(2 * maxB * p->ldA);
  p->szN = pad64(maxB * p->ldB);
  p->szW = pad64(2 * maxB * p->ldB);
  const long cap = p->cap;
  const int ns = std::max(1, pr.nslots);
  // ---- trial copies (FP32), K-major for both product directions
  const bool split = pr.passes == 3;  // also the TF32 head and tail of each copy
  const int nsec = split ? 3 : 1;
  p->to_off.resize(2 * L);
  p->tt_off.resize(2 * L);
  long nto = 0, ntt = 0;
  for (int k = 0; k < L; ++k)
    for (int s = 0; s < 2; ++s) {
      p->to_off[2 * k + s] = nto;
      nto += pad64((long)a[k + 1] * pad4(a[k]));
      p->tt_off[2 * k + s] = ntt;
      ntt += pad64((long)a[k] * pad4(a[k + 1]));
    }
  p->tos_off.resize(L);
  p->tts_off.resize(L);
  long ntos = 0, ntts = 0;
  for (int k = 0; k < L; ++k) {
    p->tos_off[k] = ntos;
    ntos += pad64((long)a[k + 1] * 2 * pad4(a[k]));
    p->tts_off[k] = ntts;
    ntts += pad64((long)a[k] * 2 * pad4(a[k + 1]));
  }
  p->nto = nto;
  p->ntt = ntt;
  p->ntos = ntos;
  p->ntts = ntts;
  int rc = palloc(p, &p->TO, nsec * nto) | palloc(p, &p->TT, nsec * ntt) | palloc(p, &p->TOs, nsec * ntos) |
           palloc(p, &p->TTs, nsec * ntts);
  if (rc) return bail(MPSQMC_E_CUDA);
  {
    std::vector<double> tr;
    long tot = 0;
    for (int k = 0; k < L; ++k) tot += 2L * a[k] * a[k + 1];
    tr.resize(tot);
    if (cudaMemcpy(tr.data(), pr.trial, sizeof(double) * tot, cudaMemcpyDeviceToHost) != cudaSuccess)
      return bail(fail(MPSQMC_E_CUDA, "batched sweep: trial download failed"));
    std::vector<float> to(nto, 0.f), tt(ntt, 0.f), tos(ntos, 0.f), tts(ntts, 0.f);
    for (int k = 0; k < L; ++k)
      for (int s = 0; s < 2; ++s) {
        const long lo = pad4(a[k]), lt = pad4(a[k + 1]);
        for (int c = 0; c < a[k + 1]; ++c)
          for (int r = 0; r < a[k]; ++r) {
            const float x = (float)tr[pr.toff[k] + r + (long)a[k] * (c + (long)a[k + 1] * s)];
            to[p->to_off[2 * k + s] + c * lo + r] = x;
            tt[p->tt_off[2 * k + s] + (long)r * lt + c] = x;
            tos[p->tos_off[k] + c * 2 * lo + s * lo + r] = x;
            tts[p->tts_off[k] + (long)r * 2 * lt + s * lt + c] = x;
          }
      }
    // sections: values, then (three passes) heads x rounded to TF32 and tails (x - head) rounded
    auto sections = [&](std::vector<float> &v) {
      const size_t n = v.size();
      if (!split) return;
      v.resize(3 * n);
      for (size_t i = 0; i < n; ++i) {
        const float h = tf32_round(v[i]);
        v[n + i] = h;
        v[2 * n + i] = tf32_round(v[i] - h);
      }
    };
    sections(to);
    sections(tt);
    sections(tos);
    sections(tts);
    if (cudaMemcpy(p->TO, to.data(), sizeof(float) * to.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->TT, tt.data(), sizeof(float) * tt.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->TOs, tos.data(), sizeof(float) * tos.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->TTs, tts.data(), sizeof(float) * tts.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(MPSQMC_E_CUDA, "batched sweep: trial upload failed"));
  }
  // ---- walker forms and right environments (site k: per walker sizes, arrays of cap walkers)
  p->sl_off.resize(L);
  p->sr_off.resize(L);
  p->sl_sz.resize(L);
  p->sr_sz.resize(L);
  p->sl_ld.resize(L);
  p->sr_ld.resize(L);
  p->r_off.resize(L + 1);
  p->r_sz.resize(L + 1);
  p->r_ld.resize(L + 1);
  long nsl = 0, nsr = 0, nr = 0;
  for (int k = 0; k < L; ++k) {
    p->sl_ld[k] = pad4(b[k]);
    p->sr_ld[k] = pad4(b[k + 1]);
    p->sl_sz[k] = pad64(2L * b[k + 1] * p->sl_ld[k]);
    p->sr_sz[k] = pad64(2L * b[k] * p->sr_ld[k]);
    p->sl_off[k] = nsl;
    p->sr_off[k] = nsr;
    nsl += p->sl_sz[k] * cap;
    nsr += p->sr_sz[k] * cap;
  }
  for (int k = 1; k <= L; ++k) {  // R_k: a_k x b_k, row-major
    p->r_ld[k] = pad4(b[k]);
    p->r_sz[k] = pad64((long)a[k] * p->r_ld[k]);
    p->r_off[k] = nr;
    nr += p->r_sz[k] * cap;
  }
  // three passes: the site forms as TF32 heads with their tails nsl (nsr) floats further on
  p->slt = split ? nsl : 0;
  p->srt = split ? nsr : 0;
  rc = palloc(p, &p->SL, (split ? 2 : 1) * nsl) | palloc(p, &p->SR, (split ? 2 : 1) * nsr) | palloc(p, &p->R, nr);
  rc |= palloc(p, &p->Lenv, p->szBl * cap) | palloc(p, &p->P, 4 * p->szBl * cap) | palloc(p, &p->X, p->szX * cap) |
        palloc(p, &p->X4, 4 * p->szX * cap) | palloc(p, &p->Y, p->szX * cap) | palloc(p, &p->Nl[0], p->szN * cap) |
        palloc(p, &p->Nl[1], p->szN * cap) | palloc(p, &p->Wn, p->szW * cap) | palloc(p, &p->Fd[0], p->szBl * cap) |
        palloc(p, &p->Fd[1], p->szBl * cap) | palloc(p, &p->Gb, 4 * p->szBl * cap) |
        palloc(p, &p->Q, pad64(2 * maxB * p->ldA) * cap) | palloc(p, &p->Fch, 3L * ns * p->szBl * cap) |
        palloc(p, &p->Xch, 3L * ns * p->szX * cap);
  // right factors written split, by class (bits of Tiles::split_out): the tails' arrays exist
  // only for the classes that are
  const int sb = split ? pr.tiles.split_out : 0;
  if (sb & kSplitY) rc |= palloc(p, &p->Yl, p->szX * cap);
  if (sb & kSplitX) rc |= palloc(p, &p->Xl, p->szX * cap);
  if (sb & kSplitX4) rc |= palloc(p, &p->X4l, 4 * p->szX * cap);
  if (sb & kSplitQ) rc |= palloc(p, &p->Ql, pad64(2 * maxB * p->ldA) * cap);
  if (sb & kSplitXch) rc |= palloc(p, &p->Xchl, 3L * ns * p->szX * cap);
  rc |= palloc(p, &p->ovb, cap) | palloc(p, &p->wtb, cap) | palloc(p, &p->scl, cap) | palloc(p, &p->ob, 8 * cap) |
        palloc(p, &p->dot, 16 * cap) | palloc(p, &p->err_tc, 1) | palloc(p, &p->nb, 1);
  if (rc) return bail(MPSQMC_E_CUDA);
  // device site tables
  {
    std::vector<int> bl(L), br(L);
    for (int k = 0; k < L; ++k) {
      bl[k] = b[k];
      br[k] = b[k + 1];
    }
    long *t_woff, *t_slo, *t_sro, *t_slz, *t_srz, *t_sll, *t_srl;
    int *t_bl, *t_br;
    rc = palloc(p, &t_woff, L) | palloc(p, &t_slo, L) | palloc(p, &t_sro, L) | palloc(p, &t_slz, L) |
         palloc(p, &t_srz, L) | palloc(p, &t_sll, L) | palloc(p, &t_srl, L) | palloc(p, &t_bl, L) | palloc(p, &t_br, L);
    if (rc) return bail(MPSQMC_E_CUDA);
    auto up = [&](void *d, const void *h, size_t n) { return cudaMemcpy(d, h, n, cudaMemcpyHostToDevice) == cudaSuccess; };
    const size_t lb = sizeof(long) * L, ib = sizeof(int) * L;
    if (!(up(t_woff, pr.woff.data(), lb) && up(t_slo, p->sl_off.data(), lb) && up(t_sro, p->sr_off.data(), lb) &&
          up(t_slz, p->sl_sz.data(), lb) && up(t_srz, p->sr_sz.data(), lb) && up(t_sll, p->sl_ld.data(), lb) &&
          up(t_srl, p->sr_ld.data(), lb) && up(t_bl, bl.data(), ib) && up(t_br, br.data(), ib)))
      return bail(fail(MPSQMC_E_CUDA, "batched sweep: table upload failed"));
    p->sf = SiteForms{t_woff, t_bl, t_br, t_slo, t_sro, t_slz, t_srz, t_sll, t_srl};
    std::vector<float> eJ(pr.ech_J.begin(), pr.ech_J.end());
    rc = palloc(p, &p->ech_slot_d, std::max<size_t>(1, pr.ech_slot.size())) |
         palloc(p, &p->ech_J_d, std::max<size_t>(1, eJ.size()));
    if (rc) return bail(MPSQMC_E_CUDA);
    if (!pr.ech_slot.empty() && !(up(p->ech_slot_d, pr.ech_slot.data(), sizeof(int) * pr.ech_slot.size()) &&
                                  up(p->ech_J_d, eJ.data(), sizeof(float) * eJ.size())))
      return bail(fail(MPSQMC_E_CUDA, "batched sweep: channel table upload failed"));
  }

  // ---- the step's launch sequence
  const Problem &q = p->pr;
  const int *ncur = q.n_cur;
  const int icap = p->cap;
  Plan *P = p;
  // a site form as an operand (with its TF32 tails when they are stored)
  auto Fm = [](Opnd o, long tail) {
    if (tail) {
      o.hi = o.base;
      o.lo = o.base + tail;
    }
    return o;
  };
  auto SLo = [P, Fm](int k) {
    return Fm(Opnd{P->SL + P->sl_off[k], P->sl_ld[k], 2L * P->pr.bW[k + 1], P->sl_sz[k], P->cap, 1}, P->slt);
  };
  auto SRo = [P, Fm](int k) {
    return Fm(Opnd{P->SR + P->sr_off[k], P->sr_ld[k], 2L * P->pr.bW[k], P->sr_sz[k], P->cap, 1}, P->srt);
  };
  auto Ro = [P](int k) { return Opnd{P->R + P->r_off[k], P->r_ld[k], P->pr.aT[k], P->r_sz[k], P->cap, 1}; };
  // a trial copy, with its head and tail sections when they exist
  auto Tr = [P, split](const float *arr, long n, long off, long ld, long rows) {
    Opnd o{arr + off, ld, rows, 0, 1, 0};
    if (split) {
      o.hi = arr + n + off;
      o.lo = arr + 2 * n + off;
    }
    return o;
  };
  auto TOo = [P, Tr](int k, int s) { return Tr(P->TO, P->nto, P->to_off[2 * k + s], pad4(P->pr.aT[k]), P->pr.aT[k + 1]); };
  auto TTo = [P, Tr](int k, int s) { return Tr(P->TT, P->ntt, P->tt_off[2 * k + s], pad4(P->pr.aT[k + 1]), P->pr.aT[k]); };
  auto TOso = [P, Tr](int k) { return Tr(P->TOs, P->ntos, P->tos_off[k], 2 * pad4(P->pr.aT[k]), P->pr.aT[k + 1]); };
  auto TTso = [P, Tr](int k) { return Tr(P->TTs, P->ntts, P->tts_off[k], 2 * pad4(P->pr.aT[k + 1]), P->pr.aT[k]); };
  // a right factor written as heads (base) with its tails at the same offset of `tails`
  auto Sp = [](Opnd o, const float *heads, const float *tails) {
    if (tails) {
      o.hi = o.base;
      o.lo = tails + (o.base - heads);
    }
    return o;
  };
  const long l2 = 2 * p->ldA;  // row stride of the unstacked right factors (X, Y as read by T3_P, T_dot)
  // sigma stride of a stacked right factor whose rows run over the trial bond a_k (K = 2 ls(k))
  auto ls = [&](int k) { return pad4((long)a[k]); };
  // right environment R_k from R_{k+1}: Y = R_{k+1} SR_k^T (rows (r, s)), then
  // R_k = sum_s TT_k[s] Y_s as one product with s stacked along K
  auto right_env = [&](int k) -> int {
    int r = add_gemm(p, Ro(k + 1), SRo(k), a[k + 1], 2 * b[k], b[k + 1], 1, p->Y, p->szX, 1, ls(k + 1), 0, 1.f, nullptr, 0,
                     0, 0, 0, 0, p->Yl);
    if (!r) {
      const Opnd Yr = Sp(Opnd{p->Y, 2 * ls(k + 1), b[k], p->szX, cap, 1}, p->Y, p->Yl);
      r = add_gemm(p, TTso(k), Yr, a[k], b[k], (int)(2 * ls(k + 1)), 1, p->R + p->r_off[k], p->r_sz[k], p->r_ld[k], 1,
                   0);
    }
    return r;
  };
  // left branches at cut i+1: X = Lenv SL_i (rows (t, c)), P[s + 2t] = TO_i[s] X_t
  auto left_branches = [&](int i) -> int {
    Opnd Le{p->Lenv, p->ldB, a[i], p->szBl, cap, 1};
    int r = add_gemm(p, Le, SLo(i), a[i], 2 * b[i + 1], b[i], 1, p->X, p->szX, 1, p->ldA, 0, 1.f, nullptr, 0, 0, 0, 0,
                     0, p->Xl);
    for (int s = 0; s < 2 && !r; ++s)
      for (int t = 0; t < 2 && !r; ++t) {
        const Opnd Xb = Sp(Opnd{p->X + (long)t * p->ldA, l2, b[i + 1], p->szX, cap, 1}, p->X, p->Xl);
        r = add_gemm(p, TOo(i, s), Xb, a[i + 1], b[i + 1], a[i], 1, p->P + (long)(s + 2 * t) * p->szBl, 4 * p->szBl,
                     p->ldB, 1, 0);
      }
    return r;
  };
  // carry the four branches through site m: X4 = P_q SL_m, P_q' = sum_s TO_m[s] X4_s
  auto carry = [&](int m) -> int {
    Opnd Pq{p->P, p->ldB, a[m], p->szBl, 4L * cap, 1};
    Opnd S = SLo(m);
    S.div = 4;
    int r = add_gemm(p, Pq, S, a[m], 2 * b[m + 1], b[m], 4, p->X4, p->szX, 1, ls(m), 0, 1.f, nullptr, 0, 0, 0, 0, 0,
                     p->X4l);
    if (!r) {
      const Opnd Xr = Sp(Opnd{p->X4, 2 * ls(m), b[m + 1], p->szX, 4L * cap, 1}, p->X4, p->X4l);
      r = add_gemm(p, TOso(m), Xr, a[m + 1], b[m + 1], (int)(2 * ls(m)), 4, p->P, p->szBl, p->ldB, 1, 0);
    }
    return r;
  };
  // closures of the branches at cut j with B_j[s'] R_{j+1} A_j[t']^T
  auto closures = [&](int j) -> int {
    double *dd = p->dot;
    const long dbytes = (long)sizeof(double) * 16 * cap;
    p->ops.push_back([dd, dbytes](cudaStream_t s, double *) {
      return cudaMemsetAsync(dd, 0, dbytes, s) == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "memset");
    });
    int r = add_gemm(p, Ro(j + 1), SRo(j), a[j + 1], 2 * b[j], b[j + 1], 1, p->Y, p->szX, 1, p->ldA, 0, 1.f, nullptr, 0,
                     0, 0, 0, 0, p->Yl);
    for (int s = 0; s < 2 && !r; ++s)
      for (int t = 0; t < 2 && !r; ++t) {
        const Opnd Yb = Sp(Opnd{p->Y + (long)t * p->ldA, l2, b[j], p->szX, cap, 1}, p->Y, p->Yl);
        r = add_gemm(p, TTo(j, s), Yb, a[j], b[j], a[j + 1], 1, p->X, 0, 0, 0, 0, 1.f, p->P, 4 * p->szBl, p->szBl,
                     p->ldB, 1, 4 * (s + 2 * t));
      }
    return r;
  };
  EnvOps eo;
  for (int k = 0; k < 4; ++k) {
    eo.opSx[k] = q.opSx[k];
    eo.opISy[k] = q.opISy[k];
    eo.opSz[k] = q.opSz[k];
  }
  SiteForms sf = p->sf;
  const int gconv = (int)std::max(1L, std::min(8L * p->sms, (2L * maxB * maxB * cap + 255) / 256));

  // step start: FP32 forms of every walker, weights, unit environments
  p->ops.push_back([=](cudaStream_t s, double *) {
    convert_kernel<<<dim3(gconv, L), 256, 0, s>>>(sf, q.walkers, q.wstride, q.slot_of, ncur, icap, P->SL, P->SR,
                                                  P->slt, P->srt);
    init_kernel<<<(icap + 255) / 256, 256, 0, s>>>(q.weight, q.slot_of, ncur, icap, P->wtb, P->Lenv, P->szBl,
                                                   P->Nl[0], P->szN, P->R + P->r_off[L], P->r_sz[L], q.err, P->nb);
    return cudaGetLastError() == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "batched sweep: start kernels");
  });
  p->launches += 2;
  for (int k = L - 1; k >= 1; --k)
    if ((rc = right_env(k))) return bail(rc);
  p->ops.push_back([=](cudaStream_t s, double *) {
    overlap0_kernel<<<(icap * 32 + 255) / 256, 256, 0, s>>>(q.trial, a[1], b[1], P->R + P->r_off[1], P->r_sz[1],
                                                            P->r_ld[1], q.walkers, q.wstride, q.slot_of, ncur, icap,
                                                            P->ovb);
    return cudaGetLastError() == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "batched sweep: overlap");
  });
  p->launches += 1;
  int rv = 1, nl = 0, fd = 0;
  std::vector<int> c0(L + 1, 0);
  for (int c = 0; c < q.nC; ++c) c0[q.ci[c] + 1] += 1;
  for (int i = 0; i < L; ++i) c0[i + 1] += c0[i];
  for (int i = 0; i < L; ++i) {
    bool kept = false;
    for (int c = c0[i]; c < c0[i + 1]; ++c) {
      const int j = q.cj[c], jq = q.cq[c];
      while (rv > j + 1) {
        --rv;
        if ((rc = right_env(rv))) return bail(rc);
      }
      if ((rc = left_branches(i))) return bail(rc);
      for (int m = i + 1; m < j; ++m)
        if ((rc = carry(m))) return bail(rc);
      if ((rc = closures(j))) return bail(rc);
      p->ops.push_back([=](cudaStream_t s, double *trace) {
        sample_kernel<<<(icap + 3) / 4, 128, 0, s>>>(P->dot, q.tabU + 16 * jq, q.tabSq + 4 * jq, q.tabVT + 16 * jq,
                                                     q.grid, q.G, q.uni, q.nC, c, ncur, icap, P->ovb, P->wtb, P->ob,
                                                     trace);
        const int g = (int)std::max(1L, std::min(8L * P->sms, ((long)std::max(b[i] * b[i + 1], b[j] * b[j + 1]) * icap + 255) / 256));
        site_op_kernel<<<dim3(g, 2), 256, 0, s>>>(sf, i, j, P->ob, q.walkers, q.wstride, q.slot_of, ncur, icap, P->SL,
                                                  P->SR, P->slt, P->srt);
        return cudaGetLastError() == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "batched sweep: sampling");
      });
      p->launches += 2;
      if (rv < j + 1) rv = j + 1;
      kept = (j == i + 1);
    }
    const int ai1 = a[i + 1], bi1 = b[i + 1];
    if (i < L - 1) {
      p->ops.push_back([=](cudaStream_t s, double *) {
        rescale_kernel<<<icap, 256, 0, s>>>(sf, i, q.walkers, q.wstride, q.slot_of, ncur, icap, P->SL, P->SR, P->slt,
                                            P->srt, P->ovb,
                                            P->scl);
        if (kept)
          derive_p_kernel<<<grid_elems(P, (long)ai1 * bi1), 256, 0, s>>>(P->P, P->szBl, P->ldB, ai1, bi1, P->ob,
                                                                         P->scl, ncur, icap);
        return cudaGetLastError() == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "batched sweep: rescale");
      });
      p->launches += kept ? 2 : 1;
      if (!kept && (rc = left_branches(i))) return bail(rc);
      // left norm environment: Nl' = sum_s C[s]^T Nl C[s]
      {
        // W = Nl SL_i (rows (c, s), ld of site i's left bond); Nl' = sum_s C[s]^T W_s in one
        // product with s stacked along K (A = site i's left form read as rows c, K = (s, m))
        const long ldl = p->sl_ld[i];
        Opnd Nlo{p->Nl[nl], p->ldB, b[i], p->szN, cap, 1};
        rc = add_gemm(p, Nlo, SLo(i), b[i], 2 * bi1, b[i], 1, p->Wn, p->szW, 1, ldl, 0);
        if (!rc) {
          const Opnd Ct = Fm(Opnd{p->SL + p->sl_off[i], 2 * ldl, bi1, p->sl_sz[i], cap, 1}, p->slt);
          Opnd Wr{p->Wn, 2 * ldl, bi1, p->szW, cap, 1};
          rc = add_gemm(p, Ct, Wr, bi1, bi1, (int)(2 * ldl), 1, p->Nl[1 - nl], p->szN, p->ldB, 1, 0);
        }
        if (rc) return bail(rc);
        nl = 1 - nl;
      }
    } else {
      if ((rc = left_branches(i))) return bail(rc);
    }
    // energy channels and the trial-walker left environment through site i
    {
      float *Fdn = p->Fdn_ptr(fd), *Fdc = p->Fd[fd];
      // the field term -h sum Sz P: written alone on site 0, added after the channel products on
      // later sites (h != 0)
      auto field_term = [=](int add) {
        P->ops.push_back([=](cudaStream_t s, double *) {
          env_init_kernel<<<grid_elems(P, (long)ai1 * bi1), 256, 0, s>>>(P->P, P->szBl, P->ldB, ai1, bi1, Fdn,
                                                                         P->szBl, P->ldB, q.h, eo, add, ncur, icap);
          return cudaGetLastError() == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "batched sweep: energy");
        });
        P->launches += 1;
      };
      if (i == 0) field_term(0);
      const int e0 = q.ech_off[i], e1 = q.ech_off[i + 1];
      int ne = 0;
      for (int e = e0; e < e1; ++e) ne += (q.ech_J[e] != 0.0) ? 1 : 0;
      if (i > 0) {
        // closing entries with J != 0, contiguous copies of (slot, J) for the kernel
        std::vector<int> es;
        std::vector<float> ej;
        for (int e = e0; e < e1; ++e)
          if (q.ech_J[e] != 0.0) {
            es.push_back(q.ech_slot[e]);
            ej.push_back((float)q.ech_J[e]);
          }
        int *es_d = nullptr;
        float *ej_d = nullptr;
        if (palloc(p, &es_d, std::max<size_t>(1, es.size())) || palloc(p, &ej_d, std::max<size_t>(1, ej.size())))
          return bail(MPSQMC_E_CUDA);
        if (!es.empty() && (cudaMemcpy(es_d, es.data(), sizeof(int) * es.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
                            cudaMemcpy(ej_d, ej.data(), sizeof(float) * ej.size(), cudaMemcpyHostToDevice) != cudaSuccess))
          return bail(fail(MPSQMC_E_CUDA, "batched sweep: channel upload failed"));
        const int ai = a[i], bi = b[i];
        const int nsl = ns;
        const long ldl = p->sl_ld[i];
        const long szQ = pad64(2 * maxB * p->ldA);
        // per sigma: G_s[t] (rows r, K = (t, c)), Q_s = sum_t G_st C[t] in one product (t along K),
        // stored Q[c (2 ldA) + s ldA + m]; then done' += sum_s TO_i[s] Q_s in one product
        p->ops.push_back([=](cudaStream_t st, double *) {
          gbuild_kernel<<<grid_elems(P, (long)ai * bi), 256, 0, st>>>(Fdc, P->szBl, P->ldB, P->Fch, P->szBl, nsl, es_d,
                                                                      ej_d, ne, ai, bi, eo, P->Gb, 4 * P->szBl,
                                                                      2 * P->szBl, ldl, ncur, icap);
          return cudaGetLastError() == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "batched sweep: energy");
        });
        p->launches += 1;
        for (int s = 0; s < 2; ++s) {
          Opnd Gr{p->Gb + 2L * s * p->szBl, 2 * ldl, ai, 4 * p->szBl, cap, 1};
          const Opnd Cr = Fm(Opnd{p->SL + p->sl_off[i], 2 * ldl, bi1, p->sl_sz[i], cap, 1}, p->slt);
          rc = add_gemm(p, Gr, Cr, ai, bi1, (int)(2 * ldl), 1, p->Q + s * ls(i), szQ, 1, 2 * ls(i), 0, 1.f, nullptr, 0,
                        0, 0, 0, 0, p->Ql ? p->Ql + s * ls(i) : nullptr);
          if (rc) return bail(rc);
        }
        const Opnd Qr = Sp(Opnd{p->Q, 2 * ls(i), bi1, szQ, cap, 1}, p->Q, p->Ql);
        rc = add_gemm(p, TOso(i), Qr, ai1, bi1, (int)(2 * ls(i)), 1, Fdn, p->szBl, p->ldB, 1, 0);
        if (rc) return bail(rc);
        if (q.h != 0.0) field_term(1);
      }
      bool cont = false;
      for (int e = e0; e < e1; ++e) cont |= q.ech_cont[e] != 0;
      if (cont) {  // every channel slot through site i (slots not open carry no data anyone reads)
        Opnd Fo{p->Fch, p->ldB, a[i], p->szBl, 3L * ns * cap, 1};
        Opnd S = SLo(i);
        S.div = 3 * ns;
        rc = add_gemm(p, Fo, S, a[i], 2 * bi1, b[i], 3 * ns, p->Xch, p->szX, 1, ls(i), 0, 1.f, nullptr, 0, 0, 0, 0, 0,
                      p->Xchl);
        if (!rc) {
          const Opnd Xr = Sp(Opnd{p->Xch, 2 * ls(i), bi1, p->szX, 3L * ns * cap, 1}, p->Xch, p->Xchl);
          rc = add_gemm(p, TOso(i), Xr, ai1, bi1, (int)(2 * ls(i)), 3 * ns, p->Fch, p->szBl, p->ldB, 1, 0);
        }
        if (rc) return bail(rc);
      }
      const int slot = q.eopen[i];
      const int nsl = ns;
      p->ops.push_back([=](cudaStream_t s, double *) {
        env_finish_kernel<<<grid_elems(P, (long)ai1 * bi1), 256, 0, s>>>(P->P, P->szBl, P->ldB, ai1, bi1, P->Lenv,
                                                                          P->szBl, P->Fch, P->szBl, nsl, slot, eo, ncur,
                                                                          icap);
        return cudaGetLastError() == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "batched sweep: energy");
      });
      p->launches += 1;
      fd = 1 - fd;
    }
  }
  // last site: energy, overlap, norm and the per-walker outputs
  {
    float *Nlc = p->Nl[nl], *Fdl = p->Fd[fd];
    const int bl = b[L - 1];
    const long wo = q.woff[L - 1];
    p->ops.push_back([=](cudaStream_t s, double *) {
      final_kernel<<<(icap * 32 + 255) / 256, 256, 0, s>>>(bl, wo, q.walkers, q.wstride, q.slot_of, Nlc, P->szN, P->ldB,
                                                          P->Lenv, P->szBl, Fdl, P->szBl, P->wtb, q.overlap, q.weight,
                                                          q.energy, q.ov_out, q.wt_out, ncur, icap, q.err);
      return cudaGetLastError() == cudaSuccess ? 0 : fail(MPSQMC_E_CUDA, "batched sweep: final");
    });
    p->launches += 1;
  }
  *out = p;
  return 0;
}

int enqueue(Plan *p, cudaStream_t stream, double *trace, int *launches) {
  for (auto &op : p->ops) {
    const int rc = op(stream, trace);
    if (rc) return rc;
  }
  if (launches) *launches = p->launches;
  return 0;
}

void destroy(Plan *p) {
  if (!p) return;
  for (void *v : p->allocs) cudaFree(v);
  delete p;
}

size_t device_bytes(const Plan *p) { return p ? p->bytes : 0; }

}  // namespace bs
}  // namespace mq
