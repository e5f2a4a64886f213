// BF16 GEMM on the 5th-generation tensor cores (tcgen05), FP32 accumulation in tensor memory.
//
//   C[m, n] = sum_k A[m, k] * B[n, k]        (A: M x K, B: N x K, both K-contiguous, "TN")
//
// One CTA computes a 128 x BN tile with 128 threads:
//   thread 0 (warp 0)  loads the K-blocks of A and B with TMA (cp.async.bulk.tensor, 128-byte
//                      swizzle) into a ring of shared-memory stages;
//   thread 32 (warp 1) issues tcgen05.mma (M = 128, N = BN, K = 16, kind::f16 with BF16 inputs)
//                      into a TMEM accumulator and frees each stage with tcgen05.commit;
//   all 4 warps        read the accumulator back with tcgen05.ld (warp w owns TMEM lanes
//                      32w..32w+31 = tile rows) and apply the epilogue.
// Every wait on an mbarrier is bounded: on timeout the CTA records an error code and skips its
// tile instead of waiting forever.
//
// Split K: grid.z > 1 gives CTA z the K-blocks [z * kb_per, (z + 1) * kb_per) and its FP32 tile
// goes to out + z * split_stride (a workspace that the caller then sums in a fixed order).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace vl {
namespace gemm {

constexpr int BM = 128;      // tile rows (UMMA M)
constexpr int BK = 64;       // K elements per stage: 128 bytes of BF16 = one swizzle row
constexpr int STAGES = 4;   // most stages of the shared-memory ring (a launch may use fewer)
constexpr unsigned kSpinLimit = 1u << 26;  // polls of an mbarrier before giving up

// Epilogue flags.
enum : int {
  EPI_ACCUM = 1,     // fp32 out: C += result (else C = result)
  EPI_BIAS = 2,      // add bias[n]
  EPI_RELU = 4,      // max(0, .)
  EPI_BF16 = 8,      // store BF16 (else FP32)
};

struct EpiParams {
  void* out;         // FP32 or BF16, row-major with leading dimension ldc
  int ldc;
  const float* bias; // length >= N
  int m_valid, n_valid;  // rows / columns of `out` to write (the padded rest is not stored)
  int flags;
  int* err;          // device error word (0 = fine)
  long long split_stride;  // elements between the partial results of consecutive K splits
  unsigned spin_limit;     // polls of an mbarrier before a wait gives up
  int drop_load;           // test hook: stage 0's A load is never issued, so every wait on it runs out
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes));
}

// Bounded wait for the phase of parity `parity` to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned limit) {
  const uint32_t addr = smem_u32(bar);
  for (unsigned it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(32);
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle: rows of 128 bytes,
// 8-row (1024-byte) swizzle atoms stacked along M/N (stride byte offset 1024), Blackwell version 1.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);         // start address, 16-byte units
  d |= (uint64_t)1u << 16;                        // leading byte offset (unused with swizzle): 1
  d |= (uint64_t)(1024u >> 4) << 32;              // stride byte offset: 1024 bytes
  d |= (uint64_t)1u << 46;                        // descriptor version (Blackwell)
  d |= (uint64_t)2u << 61;                        // layout: SWIZZLE_128B
  return d;
}

// Shared-memory matrix descriptor of an MN-major tile with 128-byte swizzle: each K row holds 64
// consecutive M (or N) values (128 bytes), 8 K rows form a 1024-byte swizzle atom; consecutive
// atoms along K are 1024 bytes apart (stride byte offset) and consecutive 64-wide column blocks
// along M / N are 64 K rows = 8192 bytes apart (leading byte offset).
#ifndef VL_MN_LBO
#define VL_MN_LBO 8192u
#endif
#ifndef VL_MN_SBO
#define VL_MN_SBO 1024u
#endif
__device__ __forceinline__ uint64_t smem_desc_sw128_mn(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((VL_MN_LBO >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((VL_MN_SBO >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// Operand layouts (kernel argument `op`): bit 0 A is MN-major (stored [K][M]), bit 1 B is
// MN-major (stored [K][N]); otherwise K-major ([M][K], [N][K]).
enum : int { OP_A_MN = 1, OP_B_MN = 2 };

// Instruction descriptor: BF16 x BF16 -> FP32, M = 128, N = bn, A / B transposed (MN-major) on
// request.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int bn, int op = 0) {
  return (1u << 4)                      // D format FP32
         | (1u << 7)                    // A format BF16
         | (1u << 10)                   // B format BF16
         | ((op & OP_A_MN) ? (1u << 15) : 0u)  // A MN-major
         | ((op & OP_B_MN) ? (1u << 16) : 0u)  // B MN-major
         | ((uint32_t)(bn >> 3) << 17)  // N >> 3
         | ((uint32_t)(BM >> 4) << 24); // M >> 4
}

template <int BN>
__global__ void __launch_bounds__(128, 1) k_gemm_bf16(const __grid_constant__ CUtensorMap tmA,
                                                      const __grid_constant__ CUtensorMap tmB, int kblocks_total,
                                                      int kb_per, int stages, int op, EpiParams ep) {
  static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "tile N");
  constexpr int A_BYTES = BM * BK * 2;
  constexpr int B_BYTES = BN * BK * 2;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment of every stage (required by the 128-byte swizzle atoms).
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  __shared__ int issued_loads;   // k-blocks whose TMA loads the producer issued

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kb_first = blockIdx.z * kb_per;
  const int kblocks = min(kblocks_total - kb_first, kb_per);   // >= 1: the host sizes the split

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    failed = 0;
    issued_loads = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;

  if (threadIdx.x == 0) {
    // TMA producer.
    int issued = 0;
    for (int kb = 0; kb < kblocks; ++kb) {
      const int s = kb % stages;
      const uint32_t round = (uint32_t)(kb / stages);
      if (!mbar_wait(&empty[s], (round & 1u) ^ 1u, ep.spin_limit)) { atomicExch(&failed, 1); break; }
      uint8_t* sa = smem + s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      const int k0 = (kb_first + kb) * BK;
      if (ep.drop_load && kb == 0) {
        // test hook: the A operand of this stage never arrives
      } else if (op & OP_A_MN) {        // two 64-row K x 64-column M boxes
        tma_load_2d(&tmA, &full[s], sa, m0, k0);
        tma_load_2d(&tmA, &full[s], sa + 8192, m0 + 64, k0);
      } else {
        tma_load_2d(&tmA, &full[s], sa, k0, m0);
      }
      if (op & OP_B_MN) {        // BN / 64 boxes of 64 K rows x 64 N columns
#pragma unroll
        for (int c = 0; c < BN / 64; ++c) tma_load_2d(&tmB, &full[s], sa + A_BYTES + 8192 * c, n0 + 64 * c, k0);
      } else {
        tma_load_2d(&tmB, &full[s], sa + A_BYTES, k0, n0);
      }
      issued = kb + 1;
    }
    issued_loads = issued;
  } else if (threadIdx.x == 32) {
    // MMA issuer.
    const uint32_t idesc = instr_desc_bf16(BN, op);
    bool ok = true;
    for (int kb = 0; kb < kblocks && ok; ++kb) {
      const int s = kb % stages;
      const uint32_t round = (uint32_t)(kb / stages);
      if (!mbar_wait(&full[s], round & 1u, ep.spin_limit)) { atomicExch(&failed, 1); ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a_addr = smem_u32(smem + s * STAGE_BYTES);
      const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
      for (int k = 0; k < BK / 16; ++k) {
        // K-major: 16 BF16 = 32 bytes further along K inside the 128-byte swizzle row;
        // MN-major: 16 K rows of 128 bytes further
        const uint64_t da = (op & OP_A_MN) ? smem_desc_sw128_mn(a_addr + 2048u * k) : smem_desc_sw128(a_addr + 32u * k);
        const uint64_t db = (op & OP_B_MN) ? smem_desc_sw128_mn(b_addr + 2048u * k) : smem_desc_sw128(b_addr + 32u * k);
        const uint32_t accumulate = (kb > 0 || k > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
      }
      // frees the stage once these MMAs have read it
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(&empty[s])));
    }
    // the accumulator is complete once every MMA issued so far has finished
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_u32(&done)));
  }

  // Epilogue: every warp waits for the accumulator, then reads its 32 rows 32 columns at a time
  // (lane = row). Each 32 x 32 block goes through shared memory (the idle stage buffers) so that
  // the global stores are row-contiguous across the warp: lane = column.
  const bool have = mbar_wait(&done, 0, ep.spin_limit);
  if (!have) atomicExch(&failed, 1);
  asm volatile("tcgen05.fence::after_thread_sync;");
  __syncthreads();   // the producer has finished issuing; every thread sees the same `failed`
  const bool good = !failed;
  if (!good && threadIdx.x == 0) {
    // Drain: whichever thread gave up, wait (bounded) for the TMA copies that may still be landing
    // in this CTA's shared memory (the last `stages` issued loads) before the block can exit.
    const int issued = issued_loads;
    for (int kb = issued > stages ? issued - stages : 0; kb < issued; ++kb)
      mbar_wait(&full[kb % stages], (uint32_t)(kb / stages) & 1u, ep.spin_limit);
  }
  if (good) {
    // the stage buffers were last read by the tensor cores (async proxy): order those reads before
    // this warp's generic writes to the same memory
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    float* stg = reinterpret_cast<float*>(smem) + warp * (32 * 33);
    const int rbase = m0 + warp * 32;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      if (n0 + c0 >= ep.n_valid) break;   // same for every warp of the CTA
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) stg[lane * 33 + j] = __uint_as_float(v[j]);
      __syncwarp();
      const int col = n0 + c0 + lane;
      const bool cok = col < ep.n_valid;
      const float bv = (cok && (ep.flags & EPI_BIAS)) ? ep.bias[col] : 0.0f;
#pragma unroll 4
      for (int r = 0; r < 32; ++r) {
        const int row = rbase + r;
        if (row >= ep.m_valid) break;     // same for every lane
        float x = stg[r * 33 + lane] + bv;
        if (ep.flags & EPI_RELU) x = fmaxf(x, 0.0f);
        if (cok) {
          const size_t o = (size_t)blockIdx.z * ep.split_stride + (size_t)row * ep.ldc + col;
          if (ep.flags & EPI_BF16) {
            ((__nv_bfloat16*)ep.out)[o] = __float2bfloat16_rn(x);
          } else if (ep.flags & EPI_ACCUM) {
            ((float*)ep.out)[o] += x;
          } else {
            ((float*)ep.out)[o] = x;
          }
        }
      }
      __syncwarp();
    }
  } else if (threadIdx.x == 0 && ep.err) {
    atomicExch(ep.err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

template <int BN>
constexpr int smem_bytes(int stages = STAGES) {
  return stages * (BM * BK * 2 + BN * BK * 2) + 1024;
}

}  // namespace gemm
}  // namespace vl
