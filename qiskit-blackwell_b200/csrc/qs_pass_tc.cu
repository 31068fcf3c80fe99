// qs_pass_tc.cu — the tile pass on the tensor cores, for dense passes.
//
// A pass whose ops are all dense two-qubit gates (Quantum-Volume circuits)
// spends its time in complex 4x4 products on the FP32 pipe: 16 FMA lanes per
// amplitude per gate, about 48 per amplitude for the three gates a 5-qubit
// register block typically holds.  Here each register block is applied as
// one 32x32 complex matrix U (its gates multiplied beforehand by
// k_block_mats, qs_pass.cu) with tcgen05.mma:
//
//   D[m][n] = sum_k X[m][k] Bt[n][k],   m = register group (128 per MMA),
//   k = 2j + (re/im) of input amplitude j, n = 2i + (re/im) of output i,
//
// so M = 128 groups, N = 64, K = 64 per block and 128 groups.  TF32 keeps 10
// mantissa bits; every FP32 operand x is split into h = x with its low 13
// bits rounded off (to nearest; exact in TF32) and l = x - h (exact in FP32),
// and D = X_l Bt_h + X_h Bt_l + X_h Bt_h accumulates in FP32 in tensor
// memory (24 MMAs of K = 8).  The dropped X_l Bt_l term and the TF32
// truncation of l leave ~3e-7 relative error per block, of either sign; the
// CUDA-core interpreter does the same work in FP32 FMAs.
//
// Per CTA (256 threads, two CTAs per SM): the tile (2^12 or 2^13 amplitudes)
// is staged in shared memory as in qs_pass.cu.  For each block and each 128
// of the tile's register groups, two threads per group each gather 16 of
// its 32 amplitudes from the tile, split them in registers and store both
// halves into the group's tensor-memory lane (tcgen05.st: the A operand
// lives in tensor memory, row m = lane m, the two threads on different
// columns); one thread issues the 24 MMAs once the block matrix (32 KiB, one
// bulk copy into shared memory) has landed, and the threads read their 16
// outputs back (tcgen05.ld) into the tile.
// Tensor memory per CTA: A high part (64 columns), A low part (64), D (64).
//
// The pass is unitary on each tile, so it keeps the tile's norm, but the
// tensor cores' FP32 accumulation truncates and shrinks it by ~3e-7 per
// block; the tile's squared norm before the first block and after the last
// (FP64) give the factor that restores it, applied as the tile is stored.
//
// Every mbarrier wait is bounded (%globaltimer); a wait that runs out ORs 8
// into the handle's status word and the kernel carries on to its end (the
// barriers stay matched, tensor memory is freed), so the host reports the
// failure through qs_device_status.
//
// Replaces, for dense passes, the per-gate dense update of the reference's
// batched QV kernel (bwk/csrc/qv8_sim_sm120.cu:58-117) and of
// apply_gate_sm120.cu:121-161.
#include "qs_api.h"
#include "qs_common.cuh"
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <set>

using namespace qs;

namespace {

// Two warpgroups: warp w works on tensor-memory lanes 32 (w % 4) .. + 31
// (register groups of those rows) and on the amplitudes 16 (w / 4) .. + 15
// of each group, i.e. on columns 32 (w / 4) .. + 31 of the A and D operands.
constexpr int kTcThreads = 256;
// Shared memory (bytes): tile | block matrix (high, low) | dep tables | S |
// mbarriers + TMEM slot | FP64 partial sums (2 per warp).
constexpr uint32_t kBOff = 65536;
constexpr uint32_t kDepOff = kBOff + 32768;
constexpr uint32_t kSOff = kDepOff + 2048;
constexpr uint32_t kBarOff = kSOff + 64;
constexpr uint32_t kRedOff = kBarOff + 32;
constexpr uint32_t kTcSmem = kRedOff + 16 * (kTcThreads / 32);
static_assert(2 * (kTcSmem + 1024) <= 228 * 1024, "tensor-core pass: two CTAs per SM");
constexpr uint32_t kMatFloats = 8192;  // one block: 4096 high + 4096 low floats
constexpr uint32_t kTmemCols = 256;    // A high (0..63), A low (64..127), D (128..191); a power of two
constexpr uint32_t kColAlo = 64, kColD = 128;

// kind::tf32 instruction descriptor: D FP32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// Tile swizzle (bank spread of the gathers), linear over GF(2): bits 1-3 of
// the amplitude index XORed with a mix of every bit from 4 up, so that the
// 32 register groups a warp gathers at once (the lowest five tile bits that
// are not register positions of the block) land on distinct banks for most
// position sets (counting the banks each warp's gather touches over the QV
// batch's blocks: 1.03x the conflict-free wavefronts, against 1.19x when bits
// 7 and 11 took no part; measured 0.5% faster).
__device__ __forceinline__ uint32_t tphys(uint32_t i) {
  return i ^ ((((i >> 4) ^ (i >> 5) ^ (i >> 7) ^ (i >> 9) ^ (i >> 11)) & 7u) << 1);
}

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t tc_timer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool tc_try(uint32_t bar, uint32_t par) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(bar), "r"(par) : "memory");
  return ok != 0u;
}
// Bounded wait for the phase of parity `par`: false once `limit` ns passed.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t par, uint64_t limit) {
  if (tc_try(bar, par)) return true;
  const uint64_t t0 = tc_timer();
  for (;;) {
    if (tc_try(bar, par)) return true;
    if (tc_timer() - t0 > limit) return false;
  }
}
// Shared-memory matrix descriptor, no swizzle, K-major canonical layout:
// 16-byte K chunks 128 bytes apart (leading byte offset), 8-row groups 2048
// bytes apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(2048u >> 4) << 32) |
         (1ull << 46);
}
// D (+)= A B with A in tensor memory (row m = lane m, K along the columns).
// The asm statements are volatile (kept in order) but clobber no memory, so
// the compiler keeps the operands in registers across the issue sequence.
__device__ __forceinline__ void tc_mma(uint32_t d, uint32_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}" ::"r"(d),
      "r"(a), "l"(b), "r"(kIdesc), "r"(acc));
}
// x rounded to the nearest TF32 value (11 significant bits; the carry of a
// round-up may move into the exponent, which is the correct result).  With
// round-to-nearest the remainder x - h takes either sign, so the truncation
// of the remainder to TF32 inside the MMA and the dropped remainder product
// do not bias amplitudes towards zero.
__device__ __forceinline__ float hi_part(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

#define TC_R8(p, b) p(v[b]), p(v[b + 1]), p(v[b + 2]), p(v[b + 3]), p(v[b + 4]), p(v[b + 5]), p(v[b + 6]), p(v[b + 7])
#define TC_OUT(x) "=r"(x)
#define TC_IN(x) "r"(x)
#define TC_REGS32                                                                                                  \
  "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, " \
  "%24, %25, %26, %27, %28, %29, %30, %31}"
#define TC_REGS32_FROM1                                                                                               \
  "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, " \
  "%25, %26, %27, %28, %29, %30, %31, %32}"
// 32 consecutive 32-bit columns of this warp's 32 tensor-memory lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 " TC_REGS32 ", [%32];"
               : TC_R8(TC_OUT, 0), TC_R8(TC_OUT, 8), TC_R8(TC_OUT, 16), TC_R8(TC_OUT, 24)
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], " TC_REGS32_FROM1 ";" ::"r"(taddr),
               TC_R8(TC_IN, 0), TC_R8(TC_IN, 8), TC_R8(TC_IN, 16), TC_R8(TC_IN, 24)
               : "memory");
}

// Sums a and b over the CTA in FP64 in a fixed order (shuffle tree within
// each warp, then the warps in index order); every thread gets the totals.
__device__ __forceinline__ void cta_sum2(double& a, double& b, double* red) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const uint32_t w = threadIdx.x >> 5;
  if ((threadIdx.x & 31u) == 0u) {
    red[2 * w] = a;
    red[2 * w + 1] = b;
  }
  __syncthreads();
  a = 0.0;
  b = 0.0;
  for (int k = 0; k < kTcThreads / 32; ++k) {
    a += red[2 * k];
    b += red[2 * k + 1];
  }
  __syncthreads();  // red is reused by the next tile
}

__global__ void __launch_bounds__(kTcThreads, 2)
k_pass_tc(float2* __restrict__ base_state, PassItem single, const PassItem* __restrict__ items, int nitems,
          uint64_t total_tiles, uint32_t* status, uint64_t limit) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* tile = reinterpret_cast<float2*>(smem);
  uint64_t* dep_lo = reinterpret_cast<uint64_t*>(smem + kDepOff);
  uint64_t* dep_hi = dep_lo + 128;
  int* s_S = reinterpret_cast<int*>(smem + kSOff);
  double* red = reinterpret_cast<double*>(smem + kRedOff);
  const uint32_t tid = threadIdx.x, warp = tid >> 5, quarter = warp & 3u, half = warp >> 2;
  const uint32_t row = 32u * quarter + (tid & 31u);  // register group (MMA row) within a 128-group slice
  const uint32_t b_bar = su32(smem + kBarOff), mma_bar = b_bar + 8u, tslot = b_bar + 16u;
  const uint32_t bhi = su32(smem + kBOff);
  // B descriptors: K step s starts 256 bytes (16 descriptor units) further
  const uint64_t bdesc_hi = tc_desc(bhi), bdesc_lo = tc_desc(bhi + 16384u);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tslot), "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b_bar), "r"(1u) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mma_bar), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + kBarOff + 16);
  const uint32_t lane = ((32u * quarter) << 16) + 32u * half;  // this warp's lanes and column half

  uint32_t nb = 0, nm = 0;  // block-matrix loads issued; MMA batches
  int cur = -1;
  const DevPass* P = nullptr;
  float2* state = nullptr;
  const float* mats = nullptr;
  int T = 0;
  for (uint64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    int it = 0;
    if (items && nitems > 1) {
      int lo = 0, hi = nitems - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].tile_begin <= t) lo = mid; else hi = mid - 1;
      }
      it = lo;
    }
    const PassItem I = items ? items[it] : single;  // a device table, else the item by value
    if (it != cur) {
      __syncthreads();  // previous tables no longer in use
      cur = it;
      P = I.pass;
      state = base_state + I.state_off;
      mats = I.mats;
      T = P->T;
      if (tid < 16) s_S[tid] = P->S[tid];
      __syncthreads();
      for (int e = tid; e < 256; e += kTcThreads) {
        const int part = e >> 7, x = e & 127;
        uint64_t d = 0;
        for (int k = 0; k < 7; ++k) {
          const int kk = part * 7 + k;
          if (kk < T && ((x >> k) & 1)) d |= 1ull << s_S[kk];
        }
        if (part == 0) dep_lo[x] = d; else dep_hi[x] = d;
      }
      __syncthreads();
    }
    const uint64_t local = t - I.tile_begin;
    uint64_t gbase = local;
    for (int k = 0; k < T; ++k) gbase = insert_zero(gbase, s_S[k]);
    const uint32_t npairs = 1u << (T - 1);
    // from |0..0>: only the tile holding index 0 of its state is non-zero
    const bool zero_tile = (I.flags & PI_FROM_ZERO) && (gbase & ((1ull << P->n_qubits) - 1ull)) != 0ull;
    if (I.flags & PI_FROM_ZERO) {
      for (uint32_t c = tid; c < npairs; c += kTcThreads) {
        const uint32_t i = c << 1;
        const float x = (!zero_tile && i == 0) ? 1.f : 0.f;
        *reinterpret_cast<float4*>(tile + tphys(i)) = make_float4(x, 0.f, 0.f, 0.f);
      }
    } else {
      for (uint32_t c = tid; c < npairs; c += kTcThreads) {
        const uint32_t i = c << 1;
        const uint64_t g = gbase | dep_lo[i & 127] | dep_hi[i >> 7];
        const uint32_t d = su32(tile + tphys(i));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(state + g) : "memory");
      }
      asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();

    const DevBlock* blocks = reinterpret_cast<const DevBlock*>(reinterpret_cast<const char*>(P) + P->block_off);
    const int nblocks = zero_tile ? 0 : P->nblocks;
    const uint32_t nmt = 1u << (T - 12);  // 128-group slices of the tile (T - 5 >= 7)
    double nin = 0.0, nout = 0.0;
    for (int b = 0; b < nblocks; ++b) {
      if (tid == 0) {
        asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(b_bar),
                     "r"(4u * kMatFloats)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(bhi),
            "l"(mats + (uint64_t)kMatFloats * b), "r"(4u * kMatFloats), "r"(b_bar)
            : "memory");
      }
      const DevBlock blk = blocks[b];
      uint32_t pp[5];
      int pos[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        pos[k] = blk.pos[k];
        pp[k] = tphys(1u << pos[k]);
      }
      const bool pair0 = pos[0] == 0;  // register bit 0 on tile bit 0
      for (uint32_t mt = 0; mt < nmt; ++mt) {
        uint32_t base = mt * 128u + row;  // group bits -> the tile's other positions, ascending
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          const uint32_t lo = base & ((1u << pos[k]) - 1u);
          base = ((base ^ lo) << 1) | lo;
        }
        // this thread's 16 amplitudes of the group: j = 16 half + j'
        uint32_t ad[16];
        ad[0] = tphys(base) ^ (half ? pp[4] : 0u);
#pragma unroll
        for (int j = 1; j < 16; ++j) ad[j] = ad[j & (j - 1)] ^ pp[__ffs(j) - 1];
        // gather (re, im interleaved = the K order); when register bit 0 is
        // tile bit 0, amplitudes j and j ^ 1 are neighbours (ad[j] is even:
        // the swizzle leaves bit 0 alone) and move as one 16-byte access
        uint32_t x[32], h[32];
        if (pair0) {
#pragma unroll
          for (int j = 0; j < 16; j += 2) {
            const float4 a = *reinterpret_cast<const float4*>(tile + ad[j]);
            x[2 * j] = __float_as_uint(a.x);
            x[2 * j + 1] = __float_as_uint(a.y);
            x[2 * j + 2] = __float_as_uint(a.z);
            x[2 * j + 3] = __float_as_uint(a.w);
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const float2 a = tile[ad[j]];
            x[2 * j] = __float_as_uint(a.x);
            x[2 * j + 1] = __float_as_uint(a.y);
          }
        }
        if (b == 0) {
#pragma unroll
          for (int e = 0; e < 32; ++e) nin = fma((double)__uint_as_float(x[e]), (double)__uint_as_float(x[e]), nin);
        }
#pragma unroll
        for (int e = 0; e < 32; e += 2) {
          const float2 v = make_float2(__uint_as_float(x[e]), __uint_as_float(x[e + 1]));
          const float2 hv = make_float2(hi_part(v.x), hi_part(v.y));
          const float2 lv = __fadd2_rn(v, make_float2(-hv.x, -hv.y));  // exact: v - hv
          h[e] = __float_as_uint(hv.x);
          h[e + 1] = __float_as_uint(hv.y);
          x[e] = __float_as_uint(lv.x);
          x[e + 1] = __float_as_uint(lv.y);
        }
        tmem_st32(tmem + lane, h);
        tmem_st32(tmem + lane + kColAlo, x);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
          if (mt == 0 && !tc_wait(b_bar, nb & 1u, limit)) atomicOr(status, 8u);
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t dcol = tmem + kColD;
#pragma unroll
          for (uint32_t s = 0; s < 8; ++s) {
            const uint64_t bh = bdesc_hi + 16u * s, bl = bdesc_lo + 16u * s;
            tc_mma(dcol, tmem + kColAlo + 8u * s, bh, s > 0 ? 1u : 0u);
            tc_mma(dcol, tmem + 8u * s, bl, 1u);
            tc_mma(dcol, tmem + 8u * s, bh, 1u);
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mma_bar)
                       : "memory");
          // the issuing thread alone waits for the MMAs; the others sleep in
          // the barrier below instead of polling (their issue slots go to
          // the SM's other CTA)
          if (!tc_wait(mma_bar, nm & 1u, limit)) atomicOr(status, 8u);
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        }
        ++nm;
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tmem_ld32(tmem + lane + kColD, x);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (b + 1 == nblocks) {
#pragma unroll
          for (int e = 0; e < 32; ++e) nout = fma((double)__uint_as_float(x[e]), (double)__uint_as_float(x[e]), nout);
        }
        if (pair0) {
#pragma unroll
          for (int j = 0; j < 16; j += 2)
            *reinterpret_cast<float4*>(tile + ad[j]) = make_float4(__uint_as_float(x[2 * j]), __uint_as_float(x[2 * j + 1]),
                                                                   __uint_as_float(x[2 * j + 2]), __uint_as_float(x[2 * j + 3]));
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            tile[ad[j]] = make_float2(__uint_as_float(x[2 * j]), __uint_as_float(x[2 * j + 1]));
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      }
      ++nb;
      __syncthreads();
    }
    float scale = 1.f;
    if (nblocks) {
      cta_sum2(nin, nout, red);
      if (nout > 0.0) scale = (float)sqrt(nin / nout);
    }
    for (uint32_t c = tid; c < npairs; c += kTcThreads) {
      const uint32_t i = c << 1;
      const uint64_t g = gbase | dep_lo[i & 127] | dep_hi[i >> 7];
      float4 v = *reinterpret_cast<const float4*>(tile + tphys(i));
      v.x *= scale;
      v.y *= scale;
      v.z *= scale;
      v.w *= scale;
      *reinterpret_cast<float4*>(state + g) = v;
    }
    __syncthreads();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

void launch_tc(qs_context* h, float2* base, const PassItem& single, const PassItem* d_items, int n_items,
               uint64_t total_tiles, int T) {
  if (n_items <= 0 || total_tiles == 0) return;
  QS_CHECK_ARG(T == 12 || T == 13, "tensor-core pass: tile bits must be 12 or 13");
  {
    static std::mutex mu;
    static std::set<int> attr_set;  // devices whose kernel attribute is set
    std::lock_guard<std::mutex> lk(mu);
    if (!attr_set.count(h->device)) {
      QS_CUDA(cudaFuncSetAttribute(k_pass_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
      attr_set.insert(h->device);
    }
  }
  const uint64_t grid = std::min<uint64_t>(total_tiles, 2ull * (uint64_t)h->sm_count);
  // a tile takes microseconds; 4 s covers time slicing with other processes
  k_pass_tc<<<(unsigned)grid, kTcThreads, kTcSmem, h->stream>>>(base, single, d_items, n_items, total_tiles,
                                                                 h->dev_status, 4000000000ull);
  qs_after_launch(h, "k_pass_tc");
}

}  // namespace

bool qs_tc_enabled(const qs_context* h) { return h && h->tensor_cores != 0; }

void qs_launch_pass_tc(qs_context* h, void* base, const PassItem* d_items, int n_items, uint64_t total_tiles, int T) {
  PassItem none{};
  launch_tc(h, static_cast<float2*>(base), none, d_items, n_items, total_tiles, T);
}

void qs_launch_pass_tc_single(qs_context* h, void* state, const DevPass* d_pass, int T, uint64_t ntiles,
                              uint32_t flags, const float* mats) {
  PassItem it{};
  it.pass = d_pass;
  it.ntiles = ntiles;
  it.flags = flags;
  it.mats = mats;
  launch_tc(h, static_cast<float2*>(state), it, nullptr, 1, ntiles, T);
}
