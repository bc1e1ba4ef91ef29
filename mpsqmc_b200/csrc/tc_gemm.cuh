// Batched FP32 products on the 5th-generation tensor cores (tcgen05, kind::tf32) for the
// walker-batched mixed-precision sweep (sm_100a).
//
//   D_z[m, n] = alpha * sum_k A_{z/adiv}[m, k] * B_{z/bdiv}[n, k]  (+ D_z[m, n] when beta)
//
// Both operands are K-major FP32 matrices (k contiguous) read by TMA (cp.async.bulk.tensor, no
// multicast, tensor maps over this GPU's memory only) into swizzled shared-memory tiles of 32
// k-values (128-byte rows, the canonical K-major SWIZZLE_128B layout of the UMMA descriptors) or
// of 16 (64-byte rows, SWIZZLE_64B: half the stage, twice the ring depth).  A divisor
// of 0 makes the operand shared by the whole batch (the trial tensor); B may stack `bstack`
// consecutive batch entries along N in one tile, so that products with a shared A become one
// wide GEMM (M = trial bond, N = walkers x walker bond).
//
// Precision: with passes = 3 every tile is split in shared memory into an exactly-TF32 head
// (x rounded to TF32) and a tail ((x - head) rounded to TF32), and the accumulator takes
// A_hi B_hi + A_hi B_lo + A_lo B_hi: about FP32 accuracy (relative error ~2^-22 per product term)
// with FP32 accumulation in TMEM.  passes = 1 runs A_hi B_hi only (TF32); bf16 runs one
// kind::f16 pass on the operands rounded to bfloat16 by the converter warps.  Operands kept in
// memory as separate head and tail arrays (the trial tensors, and outputs a product writes
// split for the next one) are loaded split: four TMA boxes per stage and no conversion, which
// takes the split's shared-memory reads and writes off the stage.
//
// Roles (384 threads, one CTA per SM, persistent over tiles):
//   warp 0      TMA producer (one lane), ring of 2-4 shared-memory stages (as many as fit);
//   warp 1      TMEM owner and MMA issuer (one lane); two or four accumulators of tn columns;
//   warps 2-7   head/tail split of each landed stage (passes = 3, operands not stored split), or
//               its rounding to bfloat16 (bf16);
//   warps 8-11  epilogue: tcgen05.ld of the accumulator (warp w reads TMEM lanes 32 (w % 4)...),
//               alpha/beta and the store to D; column-major outputs go through shared-memory
//               boxes and TMA bulk tensor stores (as head and tail arrays when the consumer
//               loads them split), row-major ones are transposed through shared memory so that
//               every store instruction writes consecutive elements.
// Every mbarrier wait is bounded: on expiry the kernel sets bit kTcErrTimeout in *err, every role
// leaves its loop, the CTA waits (bounded) for its loads in flight, frees TMEM and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace mq {
namespace tc {

constexpr int kThreads = 384;
constexpr int kMaxStages = 8;        // shared-memory stages of the load ring (2 .. 8 by tile size)
constexpr int kKC = 32;                 // k-values per stage, largest choice (128 bytes of FP32)
constexpr int kMaxTN = 256;
constexpr int kErrTimeout = 4;          // bit in the device error word (batched.h: bs::kErrTimeout)
constexpr long long kWaitCycles = 4000000000LL;  // a pipeline wait gives up after ~2 s of SM cycles

enum Epilogue : int { kStore = 0, kDot4 = 1 };
constexpr int kPassesBF16 = 16;         // mpsqmc_tc_gemm's `passes` value for one BF16 pass

struct alignas(64) GemmParams {
  CUtensorMap tmA;   // 3D (k, row, z): FP32, box (32, tm, 1), SWIZZLE_128B
  CUtensorMap tmB;   // 3D (k, row, z): FP32, box (32, brows, bstack), SWIZZLE_128B
  CUtensorMap tmD;   // dtma: D as 3D (m, n, z) with m contiguous, box (rows per epilogue warp, 16, 1)
  CUtensorMap tmA2;  // presplit: the tails of A and/or B (tmA, tmB then map the heads)
  CUtensorMap tmB2;
  CUtensorMap tmD2;  // dsplit: where the tails of D go (tmD takes the heads)
  int dtma;          // 1: column-major D (dm = 1), no accumulation: the epilogue writes through
                     // shared memory and TMA bulk tensor stores
  int presplit;      // passes = 3: bit 0 (A), bit 1 (B): the operand is stored as TF32 head and
                     // tail arrays and loaded split (no conversion of its tiles)
  int dsplit;        // dtma and passes = 3: D is written as head and tail arrays for a consumer
                     // that loads it split
  int dwide;         // dtma, not dsplit, unstacked tiles with tn a multiple of 32: tmD's box is
                     // 32 columns wide and the epilogue handles 32 columns per step
  int rtma;          // row-major D (dn = 1), no accumulation, 32-column steps that stay in one
                     // batch entry: tmD maps D as (n, m, z) with a 128-byte-swizzled box of 32
                     // columns x (rows per epilogue warp), filled with conflict-free 16-byte stores
  int M, N, K;       // per batch entry
  int tm, tn;        // MMA M (64 or 128) and tile N (multiple of 16, <= 256)
  int adiv, bdiv;    // operand batch coordinate = z / div; 0: shared (coordinate 0)
  int brows;         // B rows per batch entry loaded per tile (N when bstack > 1, else tn)
  int bstack;        // batch entries per N tile (>= 1)
  int Z;             // batch entries (if zcount: per unit of *zcount)
  const int *zcount; // optional device count: Z_total = Z * *zcount
  float alpha;
  int beta;          // 1: accumulate into D
  int passes;        // 1 or 3
  int bf16;          // 1: one BF16 pass (kind::f16): each landed FP32 stage (kc = 32) is rounded to
                     // bfloat16 into a 64-byte-swizzled copy that the products read
  int stages;        // shared-memory stages of the load ring (2 .. kMaxStages)
  int kc;            // k-values per stage: 32 (SWIZZLE_128B) or 16 (SWIZZLE_64B)
  float *D;
  long dz, dm, dn;   // D_z[m, n] = D[z dz + m dm + n dn]
  int epi;           // kStore, or kDot4: out[z] += sum_mn D_z[m,n] * E_{z,q}[m,n] for q < 4 (no store)
  const float *E;    // kDot4 operands: E_{z,q}[m, n] = E[z ez + q eq + m em + n en]
  long ez, eq, em, en;
  double *dot;       // kDot4: dot[z * dstride + doff + q], FP64 accumulation (atomic)
  int dstride, doff;
  int *err;          // device error word
};

// ---------------------------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\n"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of `parity` to complete.  Returns false (and flags the error) when
// about kWaitCycles SM cycles pass or another role already gave up.  The cycle counter is read
// only after the first 64 polls, so a wait that completes soon costs nothing beyond the polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *err) {
  unsigned n = 0;
  long long t0 = 0;
  while (!mbar_try(bar, parity)) {
    if (((++n) & 63) == 0) {
      if (*abort_flag) return false;
      const long long now = clock64();
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > kWaitCycles) {
        *abort_flag = 1;
        atomicOr(err, kErrTimeout);
        return false;
      }
    }
  }
  return true;
}

// Bounded wait used at teardown (no abort flag).
__device__ __forceinline__ void mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity) && clock64() - t0 < kWaitCycles) {
  }
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// Bulk tensor store of one shared-memory box to D at (x, y, z) (x: the contiguous coordinate;
// a multiple of 4 elements and never negative); completion tracked by the issuing thread's bulk
// groups.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int x, int y, int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
               ::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// wait until at most one committed group of this thread still reads shared memory
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
// wait until at most three committed groups of this thread still read shared memory
__device__ __forceinline__ void bulk_wait_read3() { asm volatile("cp.async.bulk.wait_group.read 3;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major, swizzled rows of 128 or 64 bytes: 8-row groups of 8 rows (stride byte offset), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t row_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                          // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((8 * row_bytes) >> 4) << 32;     // stride byte offset: one 8-row group
  d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
  d |= (uint64_t)(row_bytes == 128 ? 2 : 4) << 61;  // SWIZZLE_128B or SWIZZLE_64B
  return d;
}

// kind::tf32 (operand format 2) or kind::f16 with bfloat16 operands (format 1), FP32 accumulator,
// both operands K-major.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N, bool bf16 = false) {
  return (1u << 4) | ((bf16 ? 1u : 2u) << 7) | ((bf16 ? 1u : 2u) << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Eight consecutive FP32 values through the read-only path in one 32-byte access (p 32-byte
// aligned): a lane reads whole sectors.
__device__ __forceinline__ void ldg_v8(const float *p, float *r) {
  asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
               : "l"(p));
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------------------------
// Tile bookkeeping (identical in every role)
// ---------------------------------------------------------------------------------------------
struct Tiling {
  int mt, nt, total;  // m tiles, n tiles, all tiles
  int Zt;             // batch entries
};

__device__ __forceinline__ Tiling tiling(const GemmParams &p) {
  Tiling t;
  t.Zt = p.Z * (p.zcount ? *p.zcount : 1);
  t.mt = (p.M + p.tm - 1) / p.tm;
  if (p.bstack > 1) t.nt = (t.Zt + p.bstack - 1) / p.bstack;
  else t.nt = t.Zt * ((p.N + p.tn - 1) / p.tn);
  t.total = t.mt * t.nt;
  return t;
}

// tile -> m0, the first batch entry z0, n0 (row of B within z0; 0 when stacked)
__device__ __forceinline__ void tile_coords(const GemmParams &p, const Tiling &t, int tile, int &m0, int &z0, int &n0) {
  const int mi = tile % t.mt, ni = tile / t.mt;
  m0 = mi * p.tm;
  if (p.bstack > 1) {
    z0 = ni * p.bstack;
    n0 = 0;
  } else {
    const int per = (p.N + p.tn - 1) / p.tn;
    z0 = ni / per;
    n0 = (ni % per) * p.tn;
  }
}

// Two FP32 values rounded to bfloat16 (nearest, ties to even) and packed, the first in the low half
// (the lower k in a K-major row).
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// x rounded to the nearest TF32 value (10 explicit mantissa bits), ties away from zero, as an
// FP32 bit pattern: half of the 13 dropped bits' range is added to the magnitude bits, which are
// then cleared (a carry into the exponent is the correct rounding).  Two integer operations at
// full rate (finite x); the same values as the host's tf32_round.
__device__ __forceinline__ float to_tf32(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u);
}

// ---------------------------------------------------------------------------------------------
// The kernel
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1) tc_gemm_kernel(const __grid_constant__ GemmParams p) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ uint64_t bar_full[kMaxStages], bar_conv[kMaxStages], bar_empty[kMaxStages];
  __shared__ uint64_t bar_tfull[4], bar_tempty[4], bar_drain;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  __shared__ int issued[kMaxStages];  // loads issued per stage (for the drain at exit)

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int NS = p.stages;
  uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t row_bytes = (uint32_t)p.kc * 4;  // one tile row of kc FP32 values
  const uint32_t a_bytes = (uint32_t)p.tm * row_bytes, b_bytes = (uint32_t)p.tn * row_bytes;
  const bool bf16 = p.bf16 != 0;
  const uint32_t lo_mult = (p.passes == 3 && !bf16) ? 2u : 1u;  // head (+ tail) tiles per operand
  // BF16: [A FP32 | B FP32 | A BF16 | B BF16], the BF16 rows 64 bytes (32 values)
  const uint32_t stage_bytes = bf16 ? (a_bytes + b_bytes) * 3 / 2 : lo_mult * (a_bytes + b_bytes);
  const uint32_t b_load = (uint32_t)p.brows * p.bstack * row_bytes;  // bytes one B box brings
  const int split = (p.passes == 3 && !bf16) ? (p.presplit & 3) : 0;
  const bool conv = bf16 || (p.passes == 3 && split != 3);  // a landed stage still needs splitting
  float *stagebuf = reinterpret_cast<float *>(base + NS * stage_bytes);  // epilogue transposes
  const Tiling t = tiling(p);
  const int KC = p.kc, nk = (p.K + KC - 1) / KC;
  // accumulators in TMEM: four when they fit in its 512 columns (more slack between the products
  // of one tile and the epilogue of an earlier one), else two
  const int nacc = p.tn <= 128 ? 4 : 2;
  const int need = nacc * p.tn;
  const int tcols = need <= 32 ? 32 : (need <= 64 ? 64 : (need <= 128 ? 128 : (need <= 256 ? 256 : 512)));

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&bar_full[s], 1);
      mbar_init(&bar_conv[s], 6);
      mbar_init(&bar_empty[s], 1);
      issued[s] = 0;
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&bar_tfull[b], 1);
      mbar_init(&bar_tempty[b], 4);
    }
    mbar_init(&bar_drain, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < t.total && ok; tile += gridDim.x) {
        int m0, z0, n0;
        tile_coords(p, t, tile, m0, z0, n0);
        const int za = p.adiv ? z0 / p.adiv : 0;
        const int zb = p.bdiv ? z0 / p.bdiv : 0;
        for (int kc = 0; kc < nk; ++kc) {
          if (!mbar_wait(&bar_empty[s], ph ^ 1, &abort_flag, p.err)) {
            ok = false;
            break;
          }
          uint8_t *st = base + s * stage_bytes;
          mbar_expect_tx(&bar_full[s], ((split & 1) ? 2 : 1) * a_bytes + ((split & 2) ? 2 : 1) * b_load);
          tma_load_3d(st, &p.tmA, &bar_full[s], kc * KC, m0, za);
          tma_load_3d(st + lo_mult * a_bytes, &p.tmB, &bar_full[s], kc * KC, n0, zb);
          // tails of operands stored split, into the slots the conversion would fill
          if (split & 1) tma_load_3d(st + a_bytes, &p.tmA2, &bar_full[s], kc * KC, m0, za);
          if (split & 2) tma_load_3d(st + 2 * a_bytes + b_bytes, &p.tmB2, &bar_full[s], kc * KC, n0, zb);
          issued[s] += 1;
          if (++s == NS) {
            s = 0;
            ph ^= 1;
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int acc = 0;
      uint32_t aph = 0;  // phase bit per accumulator (a register, not an indexed array)
      const uint32_t idesc = instr_desc(p.tm, p.tn, bf16);
      bool ok = true;
      for (int tile = blockIdx.x; tile < t.total && ok; tile += gridDim.x) {
        if (!mbar_wait(&bar_tempty[acc], ((aph >> acc) & 1u) ^ 1u, &abort_flag, p.err)) break;
        tc_fence_after();
        const uint32_t dt = tmem + (uint32_t)(acc * p.tn);
        for (int kc = 0; kc < nk; ++kc) {
          uint64_t *wb = conv ? &bar_conv[s] : &bar_full[s];
          if (!mbar_wait(wb, ph, &abort_flag, p.err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          uint8_t *st = base + s * stage_bytes;
          const uint32_t ahi = smem_u32(st), alo = ahi + a_bytes, bhi = ahi + lo_mult * a_bytes, blo = bhi + b_bytes;
          if (bf16) {
            // two K = 16 products over the stage's 32 BF16 values (32 bytes apart in the row)
            const uint32_t ab = ahi + a_bytes + b_bytes, bb = ab + (uint32_t)p.tm * 64;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
              mma_bf16(dt, smem_desc(ab + kk * 32, 64), smem_desc(bb + kk * 32, 64), idesc,
                       (kc == 0 && kk == 0) ? 0u : 1u);
          }
          for (int kk = 0; kk < (bf16 ? 0 : KC / 8); ++kk) {
            const uint32_t off = kk * 32;  // 8 TF32 values = 32 bytes inside the swizzle row
            const uint32_t first = (kc == 0 && kk == 0) ? 0u : 1u;
            mma_tf32(dt, smem_desc(ahi + off, row_bytes), smem_desc(bhi + off, row_bytes), idesc, first);
            if (p.passes == 3) {
              mma_tf32(dt, smem_desc(ahi + off, row_bytes), smem_desc(blo + off, row_bytes), idesc, 1u);
              mma_tf32(dt, smem_desc(alo + off, row_bytes), smem_desc(bhi + off, row_bytes), idesc, 1u);
            }
          }
          mma_commit(&bar_empty[s]);  // frees the stage once these products are done
          if (++s == NS) {
            s = 0;
            ph ^= 1;
          }
        }
        if (!ok) break;
        mma_commit(&bar_tfull[acc]);
        aph ^= 1u << acc;
        acc = (acc + 1 == nacc) ? 0 : acc + 1;
      }
    }
  } else if (warp < 8) {
    // ---------------- head/tail split ----------------
    // head = x rounded to TF32 (cvt.rna), tail = x - head rounded to TF32: the three products
    // then miss only tail x tail and the tail's rounding (about 2^-22 relative per term)
    if (conv) {
      const int ct = threadIdx.x - 64;  // 0 .. 191
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < t.total && ok; tile += gridDim.x) {
        for (int kc = 0; kc < nk; ++kc) {
          if (!mbar_wait(&bar_full[s], ph, &abort_flag, p.err)) {
            ok = false;
            break;
          }
          uint8_t *st = base + s * stage_bytes;
          if (bf16) {
            // each 16-byte BF16 piece (8 values of a 64-byte row, swizzled by (row / 2) % 4) from
            // two 16-byte FP32 pieces of the landed 128-byte row (swizzled by row % 8)
            const int rows = p.tm + p.tn;
            uint8_t *dst = st + a_bytes + b_bytes;
            for (int v = ct; v < rows * 4; v += 192) {
              const int rr = v >> 2, c16 = v & 3;
              const bool isa = rr < p.tm;
              const int r = isa ? rr : rr - p.tm;  // row within its operand tile
              const uint8_t *src = st + (isa ? 0u : a_bytes) + (uint32_t)r * 128;
              const float4 x0 = *reinterpret_cast<const float4 *>(src + (((2 * c16) ^ (r & 7)) << 4));
              const float4 x1 = *reinterpret_cast<const float4 *>(src + (((2 * c16 + 1) ^ (r & 7)) << 4));
              uint4 o;
              o.x = pack_bf16(x0.x, x0.y);
              o.y = pack_bf16(x0.z, x0.w);
              o.z = pack_bf16(x1.x, x1.y);
              o.w = pack_bf16(x1.z, x1.w);
              uint8_t *row = dst + (isa ? 0u : (uint32_t)p.tm * 64) + (uint32_t)r * 64;
              *reinterpret_cast<uint4 *>(row + ((c16 ^ ((r >> 1) & 3)) << 4)) = o;
            }
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar_conv[s]);
            if (++s == NS) {
              s = 0;
              ph ^= 1;
            }
            continue;
          }
          // A: [hi | lo] then B: [hi | lo]; 16-byte vectors; operands loaded split are skipped
          const int na = (int)(a_bytes / 16), nb = (int)(b_bytes / 16);
          const int v0 = (split & 1) ? na : 0, v1 = (split & 2) ? na : na + nb;
          // four vectors per thread in flight: their loads issue before the first conversion
          for (int vb = v0 + ct; vb < v1; vb += 4 * 192) {
            float4 x[4];
            uint8_t *hp[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int v = vb + u * 192;
              hp[u] = (v < na) ? st + 16 * v : st + 2 * a_bytes + 16 * (v - na);
              if (v < v1) x[u] = *reinterpret_cast<float4 *>(hp[u]);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int v = vb + u * 192;
              if (v >= v1) break;
              float4 h, l;
              h.x = to_tf32(x[u].x);
              h.y = to_tf32(x[u].y);
              h.z = to_tf32(x[u].z);
              h.w = to_tf32(x[u].w);
              l.x = to_tf32(x[u].x - h.x);
              l.y = to_tf32(x[u].y - h.y);
              l.z = to_tf32(x[u].z - h.z);
              l.w = to_tf32(x[u].w - h.w);
              *reinterpret_cast<float4 *>(hp[u]) = h;
              *reinterpret_cast<float4 *>(hp[u] + ((v < na) ? a_bytes : b_bytes)) = l;
            }
          }
          fence_proxy_async();
          __syncwarp();
          if (lane == 0) mbar_arrive(&bar_conv[s]);
          if (++s == NS) {
            s = 0;
            ph ^= 1;
          }
        }
      }
    }
  } else {
    // ---------------- epilogue ----------------
    // every launch parameter the loops below use, copied to registers once: a store through D
    // may alias the parameter block as far as the compiler can tell, so reading the parameters
    // in place would repeat those loads after every store
    const int M = p.M, N = p.N, tm = p.tm, tn = p.tn, bstack = p.bstack, beta = p.beta, Zt = t.Zt;
    const int dot4 = p.epi == kDot4;
    const float alpha = p.alpha;
    float *const D = p.D;
    const long dz = p.dz, dm = p.dm, dn = p.dn;
    const float *const E = p.E;
    const long ez = p.ez, eq = p.eq, em = p.em, en = p.en;
    double *const dot = p.dot;
    const long dstride = p.dstride, doff = p.doff;
    const int NB = N * bstack;
    // every 16-column chunk lies in one batch entry (unstacked tiles, or N a multiple of 16)
    const bool chunk_uniform = bstack == 1 || (N & 15) == 0;
    const int q = warp & 3;  // TMEM lane quarter of this warp
    float *stg = stagebuf + (warp - 8) * 32 * 33;
    const bool dtma = p.dtma != 0;
    const bool staged = !dtma && !p.rtma && !dot4 && dn == 1 && dm != 1;  // row-major: transpose first
    // dtma: four 32 x 16 boxes per warp (column-major: 16 columns of nrow contiguous rows), used
    // in turn, so that up to four bulk stores per warp are in flight while the next box fills;
    // dsplit: two pairs of head and tail boxes
    const bool dsplit = dtma && p.dsplit;
    const bool dwide = dtma && p.dwide;
    const bool rtma = p.rtma != 0;
    float *dbox = stagebuf + (warp - 8) * 2048;
    int nbox = 0;
    const int nrow = (tm == 128) ? 32 : 16;            // accumulator rows this warp holds (lanes 0 .. nrow-1)
    // tile column j -> batch entry z (-1: past the stacked box, stale shared memory) and row n of B
    auto col = [&](int j, int z0, int n0, int &z, int &n) {
      if (bstack > 1) {
        z = (j < NB) ? z0 + j / N : -1;
        n = j % N;
      } else {
        z = z0;
        n = n0 + j;
      }
    };
    // closures: the lane's four partial sums (scalars, so that they stay in registers) and their
    // warp sum into entry z (one atomic per sum)
    double ds0 = 0.0, ds1 = 0.0, ds2 = 0.0, ds3 = 0.0;
    auto flush = [&](int z) {
      for (int o = 16; o > 0; o >>= 1) {
        ds0 += __shfl_xor_sync(0xffffffffu, ds0, o);
        ds1 += __shfl_xor_sync(0xffffffffu, ds1, o);
        ds2 += __shfl_xor_sync(0xffffffffu, ds2, o);
        ds3 += __shfl_xor_sync(0xffffffffu, ds3, o);
      }
      if (lane == 0) {
        double *d = dot + (long)z * dstride + doff;
        atomicAdd(d, ds0);
        atomicAdd(d + 1, ds1);
        atomicAdd(d + 2, ds2);
        atomicAdd(d + 3, ds3);
      }
      ds0 = ds1 = ds2 = ds3 = 0.0;
    };
    auto accum = [&](double x, const float *e) {
      ds0 += x * (double)e[0];
      ds1 += x * (double)e[eq];
      ds2 += x * (double)e[2 * eq];
      ds3 += x * (double)e[3 * eq];
    };
    // E rows read as 16-byte vectors when they are contiguous and aligned (chunks start at
    // columns that are multiples of 16)
    const bool e_vec = dot4 && en == 1 && ((ez | eq | em) & 3) == 0 && (reinterpret_cast<uintptr_t>(E) & 15) == 0;
    const bool e_v8 = e_vec && ((ez | eq | em) & 7) == 0 && (reinterpret_cast<uintptr_t>(E) & 31) == 0;
    int acc = 0;
    uint32_t aph = 0;
    for (int tile = blockIdx.x; tile < t.total; tile += gridDim.x) {
      int m0, z0, n0;
      tile_coords(p, t, tile, m0, z0, n0);
      if (!mbar_wait(&bar_tfull[acc], (aph >> acc) & 1u, &abort_flag, p.err)) break;
      __syncwarp();
      tc_fence_after();
      const int mq0 = m0 + (tm == 128 ? 32 * q : 16 * q);  // first row of this warp
      const int m = mq0 + lane;
      const bool mrow = lane < nrow && m < M;
      int zlast = -1;
      if (dwide) {
        // column-major output of an unstacked tile, 32 columns per step: one TMEM load, one
        // fence and one 32 x 32 bulk store amortise the loop's fixed cost (the epilogue warps
        // run one per SM sub-partition, so each step's dependent instructions are not hidden)
        for (int c0 = 0; c0 < tn; c0 += 32) {
          float v[32];
          __syncwarp();
          tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * tn + c0), v);
          const int n = n0 + c0;
          if (z0 >= Zt || n >= N) break;  // the same for every lane
          float *bx = dbox + (nbox & 1) * 1024;
          if (lane == 0) bulk_wait_read1();  // the store issued two steps ago has read bx
          __syncwarp();
          if (lane < nrow) {
#pragma unroll
            for (int i = 0; i < 32; ++i) bx[i * nrow + lane] = alpha * v[i];
          }
          fence_proxy_async();
          __syncwarp();
          if (lane == 0) {
            tma_store_3d(&p.tmD, bx, mq0, n, z0);
            bulk_commit();
          }
          ++nbox;
        }
      }
      if (rtma) {
        // row-major output, 32 columns per step: lane r writes its row's 32 values as eight
        // 16-byte pieces, piece c at position c ^ (r % 8) of the 128-byte row (the SWIZZLE_128B
        // layout the bulk store reads), so each quarter-warp's stores hit distinct banks
        for (int c0 = 0; c0 < tn; c0 += 32) {
          float v[32];
          __syncwarp();
          tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * tn + c0), v);
          int z, n;
          col(c0, z0, n0, z, n);
          if (z < 0 || z >= Zt || n >= N) break;  // later steps are past the entries too
          float *bx = dbox + (nbox & 1) * 1024;
          if (lane == 0) bulk_wait_read1();  // the store issued two steps ago has read bx
          __syncwarp();
          if (lane < nrow) {
            float4 *row = reinterpret_cast<float4 *>(bx + lane * 32);
#pragma unroll
            for (int c = 0; c < 8; ++c)
              row[c ^ (lane & 7)] = make_float4(alpha * v[4 * c], alpha * v[4 * c + 1], alpha * v[4 * c + 2],
                                                alpha * v[4 * c + 3]);
          }
          fence_proxy_async();
          __syncwarp();
          if (lane == 0) {
            tma_store_3d(&p.tmD, bx, n, mq0, z);
            bulk_commit();
          }
          ++nbox;
        }
      }
      // closures with contiguous, aligned rows of E, 32 columns per step that stay in one entry
      const bool dot_wide = dot4 && e_vec && (tn & 31) == 0 && (bstack == 1 || (N & 31) == 0);
      if (dot_wide) {
        for (int c0 = 0; c0 < tn; c0 += 32) {
          float v[32];
          __syncwarp();
          tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * tn + c0), v);
          int z, n;
          col(c0, z0, n0, z, n);
          if (z < 0 || z >= Zt || n >= N) break;  // later steps are past the entries too
          if (z != zlast) {
            if (zlast >= 0) flush(zlast);
            zlast = z;
          }
          if (!mrow) continue;
          const float *e = E + (long)z * ez + (long)m * em + (long)n;
          if (e_v8 && n + 32 <= N) {
            // whole 32-byte sectors per lane: the rows of E a warp reads are 256 bytes apart,
            // and L1 beside the stage ring is too small to keep half-read sectors
#pragma unroll
            for (int i8 = 0; i8 < 4; ++i8) {
#pragma unroll
              for (int qq = 0; qq < 4; ++qq) {
                float ev[8];
                ldg_v8(e + qq * eq + 8 * i8, ev);
                double d = 0.0;
#pragma unroll
                for (int j = 0; j < 8; ++j) d += (double)(alpha * v[8 * i8 + j]) * (double)ev[j];
                if (qq == 0) ds0 += d;
                else if (qq == 1) ds1 += d;
                else if (qq == 2) ds2 += d;
                else ds3 += d;
              }
            }
          } else if (n + 32 <= N) {
#pragma unroll
            for (int i4 = 0; i4 < 8; ++i4) {
              float4 ev[4];
#pragma unroll
              for (int qq = 0; qq < 4; ++qq) ev[qq] = __ldg(reinterpret_cast<const float4 *>(e + qq * eq) + i4);
              const double x0 = (double)(alpha * v[4 * i4]), x1 = (double)(alpha * v[4 * i4 + 1]),
                           x2 = (double)(alpha * v[4 * i4 + 2]), x3 = (double)(alpha * v[4 * i4 + 3]);
              ds0 += x0 * (double)ev[0].x + x1 * (double)ev[0].y + x2 * (double)ev[0].z + x3 * (double)ev[0].w;
              ds1 += x0 * (double)ev[1].x + x1 * (double)ev[1].y + x2 * (double)ev[1].z + x3 * (double)ev[1].w;
              ds2 += x0 * (double)ev[2].x + x1 * (double)ev[2].y + x2 * (double)ev[2].z + x3 * (double)ev[2].w;
              ds3 += x0 * (double)ev[3].x + x1 * (double)ev[3].y + x2 * (double)ev[3].z + x3 * (double)ev[3].w;
            }
          } else {
            for (int i = 0; i < 32 && n + i < N; ++i) {
              float x = v[0];
#pragma unroll
              for (int j = 1; j < 32; ++j)
                if (j == i) x = v[j];  // v[i] without an indexed (local-memory) register array
              accum((double)(alpha * x), e + i);
            }
          }
        }
      }
      for (int c0 = 0; c0 < (dwide || rtma || dot_wide ? 0 : tn); c0 += 16) {
        float v[16];
        __syncwarp();  // tcgen05.ld is warp-collective
        tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * tn + c0), v);
        int z, n;
        col(c0, z0, n0, z, n);  // the chunk's first column
        if (z < 0 || z >= Zt || n >= N) continue;  // the same for every lane
        if (chunk_uniform) {
          // all 16 columns belong to entry z, rows n .. n + nv - 1 of B: one base pointer per chunk
          const int nv = min(16, N - n);
          if (dtma) {
            // rows past M and columns past N are clipped by the tensor map's extents
            float *bx = dsplit ? dbox + (nbox & 1) * 1024 : dbox + (nbox & 3) * 512;
            if (lane == 0) {  // the stores that last used bx have read it
              if (dsplit) bulk_wait_read1();
              else bulk_wait_read3();
            }
            __syncwarp();
            if (lane < nrow) {
              if (dsplit) {  // head = x rounded to TF32, tail = (x - head) rounded to TF32
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                  const float x = alpha * v[i], h = to_tf32(x);
                  bx[i * nrow + lane] = h;
                  bx[512 + i * nrow + lane] = to_tf32(x - h);
                }
              } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) bx[i * nrow + lane] = alpha * v[i];
              }
            }
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) {
              tma_store_3d(&p.tmD, bx, mq0, n, z);
              if (dsplit) tma_store_3d(&p.tmD2, bx + 512, mq0, n, z);
              bulk_commit();
            }
            ++nbox;
            continue;
          }
          if (staged) {
            // this lane's row segment into shared memory, then lanes take the columns: each
            // store instruction writes 16 consecutive elements of each of two rows (coalesced)
#pragma unroll
            for (int i = 0; i < 16; ++i) stg[lane * 33 + i] = v[i];
            __syncwarp();
            const int cl = lane & 15, rh = lane >> 4;  // column in the chunk, row parity
            if (cl < nv) {
              float *d = D + (long)z * dz + (long)(mq0 + rh) * dm + (n + cl);
              const int rows = min(nrow, M - mq0);
              for (int r = rh; r < rows; r += 2, d += 2 * dm) {
                const float x = alpha * stg[r * 33 + cl];
                *d = beta ? *d + x : x;
              }
            }
            __syncwarp();
          } else if (!dot4) {
            if (mrow) {
              float *d = D + (long)z * dz + (long)m * dm + (long)n * dn;
#pragma unroll
              for (int i = 0; i < 16; ++i)
                if (i < nv) {
                  const float x = alpha * v[i];
                  d[i * dn] = beta ? d[i * dn] + x : x;
                }
            }
          } else {
            if (z != zlast) {
              if (zlast >= 0) flush(zlast);
              zlast = z;
            }
            if (mrow) {
              const float *e = E + (long)z * ez + (long)m * em + (long)n * en;
              if (e_vec && nv == 16) {
#pragma unroll
                for (int i4 = 0; i4 < 4; ++i4) {
                  float4 ev[4];
#pragma unroll
                  for (int qq = 0; qq < 4; ++qq) ev[qq] = __ldg(reinterpret_cast<const float4 *>(e + qq * eq) + i4);
                  const double x0 = (double)(alpha * v[4 * i4]), x1 = (double)(alpha * v[4 * i4 + 1]),
                               x2 = (double)(alpha * v[4 * i4 + 2]), x3 = (double)(alpha * v[4 * i4 + 3]);
                  ds0 += x0 * (double)ev[0].x + x1 * (double)ev[0].y + x2 * (double)ev[0].z + x3 * (double)ev[0].w;
                  ds1 += x0 * (double)ev[1].x + x1 * (double)ev[1].y + x2 * (double)ev[1].z + x3 * (double)ev[1].w;
                  ds2 += x0 * (double)ev[2].x + x1 * (double)ev[2].y + x2 * (double)ev[2].z + x3 * (double)ev[2].w;
                  ds3 += x0 * (double)ev[3].x + x1 * (double)ev[3].y + x2 * (double)ev[3].z + x3 * (double)ev[3].w;
                }
              } else {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                  if (i < nv) accum((double)(alpha * v[i]), e + i * en);
              }
            }
          }
          continue;
        }
        // a chunk that spans two batch entries (stacked tiles with N not a multiple of 16): per element
        if (staged) {
#pragma unroll
          for (int i = 0; i < 16; ++i) stg[lane * 33 + i] = v[i];
          __syncwarp();
          const int cl = lane & 15, rh = lane >> 4;
          int zc, nc;
          col(c0 + cl, z0, n0, zc, nc);
          if (zc >= 0 && zc < Zt && nc < N) {
            float *dcol = D + (long)zc * dz + nc;
            for (int r = rh; r < nrow; r += 2) {
              const int mm = mq0 + r;
              if (mm < M) {
                float *d = dcol + (long)mm * dm;
                const float x = alpha * stg[r * 33 + cl];
                *d = beta ? *d + x : x;
              }
            }
          }
          __syncwarp();
        } else if (!dot4) {
          if (mrow) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              int zi, ni;
              col(c0 + i, z0, n0, zi, ni);
              if (zi < 0 || zi >= Zt || ni >= N) continue;
              float *d = D + (long)zi * dz + (long)m * dm + (long)ni * dn;
              const float x = alpha * v[i];
              *d = beta ? *d + x : x;
            }
          }
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            int zi, ni;
            col(c0 + i, z0, n0, zi, ni);
            if (zi < 0 || zi >= Zt || ni >= N) continue;
            if (zi != zlast) {
              if (zlast >= 0) flush(zlast);
              zlast = zi;
            }
            if (mrow) accum((double)(alpha * v[i]), E + (long)zi * ez + (long)m * em + (long)ni * en);
          }
        }
      }
      if (dot4 && zlast >= 0) flush(zlast);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bar_tempty[acc]);
      aph ^= 1u << acc;
      acc = (acc + 1 == nacc) ? 0 : acc + 1;
    }
    // the bulk stores this warp issued have completed (they read its boxes until then)
    if ((dtma || rtma) && lane == 0) bulk_wait_all();
  }

  // ---------------- teardown ----------------
  __syncthreads();
  if (threadIdx.x == 0 && abort_flag) {
    // the loads issued into each stage complete its full barrier in order: wait (bounded) for
    // the last one, so that no copy lands in shared memory after the CTA has gone
    for (int s = 0; s < NS; ++s) {
      if (issued[s] == 0) continue;
      mbar_wait_bounded(&bar_full[s], (uint32_t)((issued[s] - 1) & 1));
    }
  }
  if (warp == 1 && lane == 0) {
    // every product this CTA issued has finished writing TMEM before it is freed
    mma_commit(&bar_drain);
    mbar_wait_bounded(&bar_drain, 0);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols));
  }
}

// Shared memory of one launch: the stage ring (head and, with 3 passes, tail tiles), the
// epilogue's transpose buffers and the 1024-byte alignment slack.
__host__ __device__ constexpr int stage_bytes_of(int tm, int tn, int passes, int kc = kKC, int bf16 = 0) {
  return bf16 ? (tm + tn) * kc * 6 : (passes == 3 ? 2 : 1) * (tm + tn) * kc * 4;
}
// The epilogue's staging area: transposes (4 warps x 32 x 33 floats) or store boxes (4 warps x
// 4 boxes of 32 x 16 floats, or two pairs of head and tail boxes).
__host__ __device__ constexpr int staging_bytes(int dsplit) { return 4 * 2048 * 4 + 0 * dsplit; }
__host__ __device__ constexpr int smem_bytes(int tm, int tn, int passes, int stages, int dsplit = 0, int kc = kKC,
                                            int bf16 = 0) {
  return stages * stage_bytes_of(tm, tn, passes, kc, bf16) + staging_bytes(dsplit) + 1024;
}
// As many stages (2 .. kMaxStages) as fit in the opt-in shared memory.
inline int stages_for(int tm, int tn, int passes, int smem_limit, int dsplit = 0, int kc = kKC, int bf16 = 0) {
  int s = kMaxStages;
  while (s > 2 && smem_bytes(tm, tn, passes, s, dsplit, kc, bf16) > smem_limit) --s;
  return s;
}


}  // namespace tc
}  // namespace mq
