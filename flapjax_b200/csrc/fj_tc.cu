// fj_tc.cu -- tensor-core GEMM for the mixed-precision factorisation (sm_100a tcgen05).
//
// C <- alpha * A B + beta * C with A (m x k) and B (k x n) row-major FP32.  One CTA owns a
// 128 x 128 tile of C; its accumulator lives in tensor memory (128 lanes x 128 FP32
// columns).  Operands go through shared memory in the K-major 128-byte-swizzle layout the
// MMA descriptors name: a 128-row x 32-float slab per tile, row r at r * 128 bytes, the
// 16-byte chunk c of a row stored at chunk position c ^ (r & 7).  The CTA stages slabs
// itself (coalesced loads; B transposed on the way in), so any leading dimension works.
//
// Precision: an FP32 value x splits into hi = rna_tf32(x) and lo = x - hi (exact).  With
// passes = 3 the tile accumulates hi*hi + hi*lo + lo*hi (the dropped lo*lo term is
// below 2^-22 |x||y|), so the product keeps close to FP32 accuracy on the TF32 pipe; with
// passes = 1 it is a plain TF32 product (hi*hi).
//
// Synchronisation: one elected thread issues tcgen05.mma and commits each slab's MMAs to
// an mbarrier; the CTA waits on it before refilling that slab's buffer and before the
// epilogue.  Every wait is bounded (about one second); on expiry the CTA records the
// failure in *err, drains its MMAs with a second bounded wait, frees its tensor memory
// and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "fj_tc.cuh"

namespace fj {
namespace {

constexpr int kBM = 128, kBN = 128;  // C tile
constexpr int kBK = 32;               // floats per 128-byte swizzle row = one K slab
constexpr int kThreads = 256;
constexpr int kSlabBytes = kBM * kBK * 4;    // 16 KB (A and B slabs alike, kBN == kBM)
constexpr int kStageBytes = 4 * kSlabBytes;  // A hi, A lo, B hi, B lo
constexpr int kStages = 2;
constexpr size_t kGemmSmem = (size_t)kStages * kStageBytes + 1024;  // + alignment slack
constexpr uint32_t kTmemCols = 128;
constexpr long long kWaitCycles = 2000000000ll;  // ~1 s at the B200 SM clock

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (tcgen05): K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart.  Start address and offsets are in 16-byte units.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;            // leading-dimension offset (unused for this layout)
    d |= (uint64_t)(1024 >> 4) << 32;  // stride-dimension offset: one 8-row group
    d |= (uint64_t)1 << 46;            // descriptor version
    d |= (uint64_t)2 << 61;            // swizzle mode: 128 B
    return d;
}

// Instruction descriptor: D FP32, A and B TF32, both K-major, M = kBM, N = kBN.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the completion of phase `parity`; false when the bound expired.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!bar_try_wait(bar, parity))
        if (clock64() - t0 > kWaitCycles) return false;
    return true;
}

__device__ __forceinline__ float tf32_hi(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Byte offset of element (row, kk) of a swizzled slab (row < 128, kk < 32).
__device__ __forceinline__ uint32_t swz(int row, int kk) {
    return (uint32_t)(row * 128 + ((((kk >> 2) ^ (row & 7)) << 4) | ((kk & 3) << 2)));
}

// One K slab of both operands in registers: 16 floats of A and 16 of B per thread.
//   A (rows m0.., columns k0..k0+31): lane = k, the warp's rows every 8th row, so a warp
//     load is 32 consecutive floats of one row.
//   B (rows k0..k0+31, columns n0..): thread = column, four consecutive k per 16-byte
//     chunk; every load is coalesced across the warp's consecutive columns.
// All 32 loads are issued before any use, so one slab costs one memory round trip.
struct Slab {
    float a[16];
    float b[16];
};

__device__ __forceinline__ void load_slab(Slab& r, const float* a, int lda, const float* b, int ldb, int m, int n,
                                          int k, int m0, int n0, int k0) {
    const int gk = k0 + (threadIdx.x & 31);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int gm = m0 + (threadIdx.x >> 5) + 8 * i;
        r.a[i] = (gm < m && gk < k) ? __ldg(a + (int64_t)gm * lda + gk) : 0.0f;
    }
    const int gn = n0 + (threadIdx.x & (kBN - 1));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int c4 = (threadIdx.x / kBN) + 2 * i;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gkb = k0 + c4 * 4 + j;
            r.b[i * 4 + j] = (gkb < k && gn < n) ? __ldg(b + (int64_t)gkb * ldb + gn) : 0.0f;
        }
    }
}

// Registers -> the swizzled K-major slabs (hi, and lo when split).  A: a warp writes 32
// distinct banks; B: 16-byte chunks, eight consecutive columns on distinct chunk slots.
__device__ __forceinline__ void store_slab(const Slab& r, unsigned char* base, bool split) {
    unsigned char* a_hi = base;
    unsigned char* a_lo = base + kSlabBytes;
    unsigned char* b_hi = base + 2 * kSlabBytes;
    unsigned char* b_lo = base + 3 * kSlabBytes;
    const int kk = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int row = (threadIdx.x >> 5) + 8 * i;
        const uint32_t off = swz(row, kk);
        const float h = tf32_hi(r.a[i]);
        *reinterpret_cast<float*>(a_hi + off) = h;
        if (split) *reinterpret_cast<float*>(a_lo + off) = r.a[i] - h;
    }
    const int col = threadIdx.x & (kBN - 1);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int c4 = (threadIdx.x / kBN) + 2 * i;
        const float4 x = make_float4(r.b[4 * i], r.b[4 * i + 1], r.b[4 * i + 2], r.b[4 * i + 3]);
        const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
        const uint32_t off = (uint32_t)(col * 128 + ((c4 ^ (col & 7)) << 4));
        *reinterpret_cast<float4*>(b_hi + off) = h;
        if (split) *reinterpret_cast<float4*>(b_lo + off) = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
    }
}

__global__ void __launch_bounds__(kThreads, 1)
    tc_gemm_tf32_kernel(const float* a, int lda, const float* b, int ldb, float* c, int ldc, int m, int n,
                        int k, float alpha, float beta, int passes, int* __restrict__ err) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[kStages];
    __shared__ uint32_t s_tmem;
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    const bool split = passes == 3;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[s])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    const int n_slab = (k + kBK - 1) / kBK;
    bool ok = true;
    int issued = 0;  // slabs whose MMAs were committed
    Slab regs;
    load_slab(regs, a, lda, b, ldb, m, n, k, m0, n0, 0);
    for (int ks = 0; ks < n_slab; ++ks) {
        const int st = ks & 1;
        unsigned char* base = smem + st * kStageBytes;
        if (ks >= kStages) {  // the MMAs of slab ks-2 read this buffer
            const bool w = bar_wait(&bars[st], (uint32_t)(((ks - kStages) >> 1) & 1));
            ok = __syncthreads_and(w) != 0;
            if (!ok) break;
        }
        store_slab(regs, base, split);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // the next slab's loads are in flight while this slab's MMAs run
        if (ks + 1 < n_slab) load_slab(regs, a, lda, b, ldb, m, n, k, m0, n0, (ks + 1) * kBK);
        if (threadIdx.x == 0 && passes != 0) {  // passes = 0: the wait self-test issues nothing
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(base), sb = smem_u32(base + 2 * kSlabBytes);
#pragma unroll
            for (int kk = 0; kk < kBK / 8; ++kk) {  // K = 8 per tf32 MMA = 32 bytes
                const uint32_t step = (uint32_t)kk * 32u;
                const uint64_t ah = sw128_desc(sa + step), bh = sw128_desc(sb + step);
                mma_tf32(tmem, ah, bh, (ks > 0 || kk > 0) ? 1u : 0u);
                if (split) {
                    const uint64_t al = sw128_desc(sa + kSlabBytes + step);
                    const uint64_t bl = sw128_desc(sb + kSlabBytes + step);
                    mma_tf32(tmem, ah, bl, 1u);
                    mma_tf32(tmem, al, bh, 1u);
                }
            }
            mma_commit(&bars[st]);
        }
        issued = ks + 1;
    }
    // this thread's C values for the epilogue, loaded while the last MMAs run: rows
    // m0 + 32 (w%4) + r, column n0 + 64 (w/4) + 32 cc + lane
    const int q = warp & 3, h = warp >> 2;
    float cpre[2][32];
    if (beta != 0.0f) {
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int col = n0 + 64 * h + 32 * cc + lane;
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const int row = m0 + 32 * q + r;
                cpre[cc][r] = (row < m && col < n) ? c[(int64_t)row * ldc + col] : 0.0f;
            }
        }
    }
    if (issued > 0) {  // all MMAs done: the last commit covers every earlier one
        const int last = issued - 1;
        const bool w = bar_wait(&bars[last & 1], (uint32_t)((last >> 1) & 1));
        const bool all = __syncthreads_and(w) != 0;
        if (!all) ok = false;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && issued == n_slab && n_slab > 0) {
        // warp w reads TMEM lanes 32*(w%4).. (tile rows) and columns 64*(w/4)..+63; each
        // 32 x 32 block goes through the warp's own padded shared-memory square (the
        // operand buffers are idle now) so that C is read and written row by row, coalesced
        float* sq = reinterpret_cast<float*>(smem) + warp * (32 * 33);
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int col0 = 64 * h + 32 * cc;
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)col0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                  "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                  "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                  "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 32; ++j) sq[lane * 33 + j] = __uint_as_float(v[j]);  // row lane, column j
            __syncwarp();
            const int col = n0 + col0 + lane;
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const int row = m0 + 32 * q + r;
                if (row < m && col < n) {
                    const float acc = alpha * sq[r * 33 + lane];
                    c[(int64_t)row * ldc + col] = beta != 0.0f ? acc + beta * cpre[cc][r] : acc;
                }
            }
            __syncwarp();
        }
    } else if (!ok && threadIdx.x == 0) {
        *err = 1;
        // drain: a second bounded wait on the last committed slab before freeing TMEM
        if (issued > 0) (void)bar_wait(&bars[(issued - 1) & 1], (uint32_t)(((issued - 1) >> 1) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// Inverses of 128 x 128 diagonal blocks of packed LU factors, one CTA per block
// b = b0 + blockIdx.x: the unit lower triangle, or (upper) the upper triangle with its
// diagonal.  A block (ib <= 128 rows at i0 = 128 b) is padded to 128 with the identity and
// inverted by doubling: at block size s each pair of inverted s x s diagonal blocks yields
// the off-diagonal block of their 2s x 2s inverse, X21 = -X22 (L21 X11) for lower and
// X12 = -X11 (U12 X22) for upper.  Output: out + 128*128*b, row-major, zero outside the
// ib x ib block.
constexpr int kTriS = 129;  // padded shared-memory row stride (floats)
constexpr size_t kTriSmem = (size_t)(2 * 128 * kTriS + 64 * 128) * sizeof(float);

__global__ void __launch_bounds__(512) tri_inv_kernel(const float* __restrict__ lu, int n, int b0, bool upper,
                                                      float* __restrict__ out_all) {
    extern __shared__ float tri_sm[];
    float* Ls = tri_sm;
    float* Xs = Ls + 128 * kTriS;
    float* Ts = Xs + 128 * kTriS;  // 64 * 128 floats: every pair's s x s product at level s
    const int b = b0 + blockIdx.x;
    const int i0 = b * 128, ib = min(128, n - i0);
    float* out = out_all + (size_t)b * 128 * 128;
#pragma unroll 16
    for (int idx = threadIdx.x; idx < 128 * 128; idx += blockDim.x) {
        const int r = idx >> 7, c = idx & 127;
        float v = (r == c) ? 1.0f : 0.0f;
        if (r < ib && c < ib) {
            if (upper ? (c >= r) : (c < r)) v = lu[(int64_t)(i0 + r) * n + i0 + c];
        }
        Ls[r * kTriS + c] = v;
        Xs[r * kTriS + c] = (r == c) ? (upper ? 1.0f / v : 1.0f) : 0.0f;
    }
    __syncthreads();
    for (int s = 1; s < 128; s <<= 1) {
        const int ss = s * s, work = (128 / (2 * s)) * ss;
        for (int idx = threadIdx.x; idx < work; idx += blockDim.x) {
            const int pi = idx / ss, rc = idx - pi * ss, r = rc / s, c = rc - r * s;
            const int p = pi * 2 * s;
            float acc = 0.0f;
            if (!upper) {
                for (int t = c; t < s; ++t) acc += Ls[(p + s + r) * kTriS + p + t] * Xs[(p + t) * kTriS + p + c];
            } else {
                for (int t = 0; t <= c; ++t)
                    acc += Ls[(p + r) * kTriS + p + s + t] * Xs[(p + s + t) * kTriS + p + s + c];
            }
            Ts[idx] = acc;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < work; idx += blockDim.x) {
            const int pi = idx / ss, rc = idx - pi * ss, r = rc / s, c = rc - r * s;
            const int p = pi * 2 * s;
            const float* T = Ts + pi * ss;
            float acc = 0.0f;
            if (!upper) {
                for (int t = 0; t <= r; ++t) acc += Xs[(p + s + r) * kTriS + p + s + t] * T[t * s + c];
                Xs[(p + s + r) * kTriS + p + c] = -acc;
            } else {
                for (int t = r; t < s; ++t) acc += Xs[(p + r) * kTriS + p + t] * T[t * s + c];
                Xs[(p + r) * kTriS + p + s + c] = -acc;
            }
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < 128 * 128; idx += blockDim.x) {
        const int r = idx >> 7, c = idx & 127;
        out[idx] = (r < ib && c < ib) ? Xs[r * kTriS + c] : 0.0f;
    }
}

// ---------------------------------------------------------------------------------
// TMA-fed form, for the products of the factorisation.  The operands are first split
// into TF32 hi (and lo) copies, A as (m x kp) and B transposed as (n x kp), K contiguous
// and padded to whole 32-float slabs (tc_split_*_kernel), so that every slab is a
// 128-row x 128-byte box a TMA load brings in already in the 128-byte-swizzled K-major
// layout the MMA descriptors name.  Roles, 4 warps: lane 0 of warp 0 loads (cp.async.bulk
// .tensor, no multicast) into a ring of kTmaStages slab stages, each completing a "full"
// mbarrier by its transaction bytes; lane 0 of warp 1 waits on "full", issues the slab's
// MMAs and commits them to the stage's "empty" mbarrier, which frees the stage for the
// producer; after the last slab it commits to "done".  All eight warps read their share
// of C into registers before the main loop (beta != 0), wait on "done", and write the
// tile (TMEM -> registers -> a warp's shared-memory square -> C, coalesced).
// Every wait is bounded (about one second); on expiry the CTA records the failure in
// *err, waits (bounded) for the loads it issued, frees its tensor memory and returns
// without writing C.
constexpr int kTmaThreads = 256;
constexpr int kTmaStages = 3;
constexpr size_t kTmaSmem = (size_t)kTmaStages * kStageBytes + 1024;

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// One box of a 2D tensor map (x = element column, y = row) into shared memory; the load
// completes its bytes on *bar.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__global__ void __launch_bounds__(kTmaThreads, 1)
    tc_gemm_tma_kernel(const __grid_constant__ CUtensorMap ta_hi, const __grid_constant__ CUtensorMap ta_lo,
                       const __grid_constant__ CUtensorMap tb_hi, const __grid_constant__ CUtensorMap tb_lo,
                       float* c, int ldc, int m, int n, int kp, float alpha, float beta, int passes,
                       int* __restrict__ err) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[kTmaStages], empty[kTmaStages], done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail, s_loaded, s_used;
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    const bool split = passes == 3;
    const uint32_t stage_tx = (split ? 4u : 2u) * (uint32_t)kSlabBytes;
    const int n_slab = kp / kBK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int st = 0; st < kTmaStages; ++st) {
            bar_init(&full[st], 1);
            bar_init(&empty[st], 1);
        }
        bar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
        s_loaded = 0;
        s_used = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // this thread's C values for the epilogue: rows m0 + 32 (w%4) + r, columns
    // n0 + 64 (w/4) + 32 cc + lane; the loads fly while the tile is computed
    const int q = warp & 3, hc = warp >> 2;
    float cpre[2][32];
    if (beta != 0.0f) {
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int col = n0 + 64 * hc + 32 * cc + lane;
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const int row = m0 + 32 * q + r;
                cpre[cc][r] = (row < m && col < n) ? c[(int64_t)row * ldc + col] : 0.0f;
            }
        }
    }

    if (warp == 0 && lane == 0) {  // producer
        int loaded = 0;
        for (int ks = 0; ks < n_slab; ++ks) {
            const int st = ks % kTmaStages;
            if (ks >= kTmaStages && !bar_wait(&empty[st], (uint32_t)(((ks - kTmaStages) / kTmaStages) & 1))) {
                s_fail = 1;
                break;
            }
            unsigned char* base = smem + st * kStageBytes;
            bar_expect_tx(&full[st], stage_tx);
            tma_load_2d(base, &ta_hi, ks * kBK, m0, &full[st]);
            tma_load_2d(base + 2 * kSlabBytes, &tb_hi, ks * kBK, n0, &full[st]);
            if (split) {
                tma_load_2d(base + kSlabBytes, &ta_lo, ks * kBK, m0, &full[st]);
                tma_load_2d(base + 3 * kSlabBytes, &tb_lo, ks * kBK, n0, &full[st]);
            }
            loaded = ks + 1;
        }
        s_loaded = loaded;
    } else if (warp == 1 && lane == 0) {  // MMA issuer
        int used = 0;
        for (int ks = 0; ks < n_slab; ++ks) {
            const int st = ks % kTmaStages;
            if (!bar_wait(&full[st], (uint32_t)((ks / kTmaStages) & 1))) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            unsigned char* base = smem + st * kStageBytes;
            const uint32_t sa = smem_u32(base), sb = smem_u32(base + 2 * kSlabBytes);
#pragma unroll
            for (int kk = 0; kk < kBK / 8; ++kk) {
                const uint32_t step = (uint32_t)kk * 32u;
                const uint64_t ah = sw128_desc(sa + step), bh = sw128_desc(sb + step);
                mma_tf32(tmem, ah, bh, (ks > 0 || kk > 0) ? 1u : 0u);
                if (split) {
                    mma_tf32(tmem, ah, sw128_desc(sb + kSlabBytes + step), 1u);
                    mma_tf32(tmem, sw128_desc(sa + kSlabBytes + step), bh, 1u);
                }
            }
            mma_commit(&empty[st]);
            used = ks + 1;
        }
        mma_commit(&done);  // arrives once every MMA issued above has completed
        s_used = used;
    }
    const bool w = bar_wait(&done, 0u);
    const bool all = __syncthreads_and(w) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool ok = all && s_fail == 0 && s_used == n_slab;
    if (ok) {
        // warp w reads TMEM lanes 32 (w%4).. (tile rows) and columns 64 (w/4)..+63
        float* sq = reinterpret_cast<float*>(smem) + warp * (32 * 33);
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int col0 = 64 * hc + 32 * cc;
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)col0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                  "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                  "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                  "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 32; ++j) sq[lane * 33 + j] = __uint_as_float(v[j]);  // row lane, column j
            __syncwarp();
            const int col = n0 + col0 + lane;
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const int row = m0 + 32 * q + r;
                if (row < m && col < n) {
                    const float acc = alpha * sq[r * 33 + lane];
                    c[(int64_t)row * ldc + col] = beta != 0.0f ? acc + beta * cpre[cc][r] : acc;
                }
            }
            __syncwarp();
        }
    } else if (threadIdx.x == 0) {
        *err = 1;
        // the loads issued and not consumed still land in shared memory: wait for them
        for (int ks = s_used; ks < s_loaded; ++ks)
            (void)bar_wait(&full[ks % kTmaStages], (uint32_t)((ks / kTmaStages) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// hi (and lo) TF32 copies of both operands in one launch.  CTAs [0, n_row_ctas): A (m x k,
// lda) as (m x kp), columns k..kp zero, grid-stride.  The rest: B (k x n, ldb) transposed
// to (n x kp), one 32 x 32 tile per CTA through shared memory (tile t: columns
// 32 (t % tiles_n), rows 32 (t / tiles_n) of B).
__global__ void __launch_bounds__(256) tc_split_kernel(const float* __restrict__ a, int lda, int m,
                                                       const float* __restrict__ b, int ldb, int n, int k, int kp,
                                                       float* __restrict__ a_hi, float* __restrict__ a_lo,
                                                       float* __restrict__ b_hi, float* __restrict__ b_lo,
                                                       int n_row_ctas) {
    if ((int)blockIdx.x < n_row_ctas) {
        const int64_t total = (int64_t)m * kp;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
             i += (int64_t)n_row_ctas * blockDim.x) {
            const int r = (int)(i / kp), cc = (int)(i % kp);
            const float v = cc < k ? a[(int64_t)r * lda + cc] : 0.0f;
            const float h = tf32_hi(v);
            a_hi[i] = h;
            if (a_lo) a_lo[i] = v - h;
        }
        return;
    }
    __shared__ float t[32][33];
    const int tiles_n = (n + 31) / 32;
    const int tile = (int)blockIdx.x - n_row_ctas;
    const int j0 = (tile % tiles_n) * 32, k0 = (tile / tiles_n) * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {  // rows of B: k0 + r, columns j0 + tx
        const int kk = k0 + r, j = j0 + tx;
        t[r][tx] = (kk < k && j < n) ? b[(int64_t)kk * ldb + j] : 0.0f;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {  // rows of the copy: j0 + r, columns k0 + tx
        const int j = j0 + r, kk = k0 + tx;
        if (j < n) {
            const float v = t[tx][r];
            const float h = tf32_hi(v);
            b_hi[(int64_t)j * kp + kk] = h;
            if (b_lo) b_lo[(int64_t)j * kp + kk] = v - h;
        }
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

// A row-major (rows x kp) FP32 matrix as 128-row x 32-float boxes, 128-byte swizzle.
static bool encode_slabs(CUtensorMap* map, const float* base, int rows, int kp) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kp * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kBM};
    const cuuint32_t elem[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, elem,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

int tc_gemm_tf32(const float* a, int lda, const float* b, int ldb, float* c, int ldc, int m, int n, int k,
                 float alpha, float beta, int passes, int* d_err, cudaStream_t s) {
    if (m < 0 || n < 0 || k <= 0 || lda < k || ldb < n || ldc < n)
        return fail(FJ_ERR_SHAPE, "tc_gemm: m=%d n=%d k=%d lda=%d ldb=%d ldc=%d", m, n, k, lda, ldb, ldc);
    if (passes != 1 && passes != 3) return fail(FJ_ERR_SHAPE, "tc_gemm: passes=%d (1 or 3)", passes);
    if (m == 0 || n == 0) return FJ_OK;
    FJ_TRY(allow_dynamic_smem((const void*)tc_gemm_tf32_kernel, kGemmSmem));
    dim3 grid((unsigned)((n + kBN - 1) / kBN), (unsigned)((m + kBM - 1) / kBM));
    tc_gemm_tf32_kernel<<<grid, kThreads, kGemmSmem, s>>>(a, lda, b, ldb, c, ldc, m, n, k, alpha, beta, passes, d_err);
    note_launch();
    FJ_LAUNCH_CHECK("tc_gemm_tf32_kernel");
    return FJ_OK;
}

size_t tc_gemm_scratch_floats(int m, int n, int k, int passes) {
    const size_t kp = (size_t)((k + kBK - 1) / kBK) * kBK;
    return (size_t)(m + n) * kp * (passes == 3 ? 2 : 1);
}

int tc_gemm_tf32_tma(const float* a, int lda, const float* b, int ldb, float* c, int ldc, int m, int n, int k,
                     float alpha, float beta, int passes, float* scratch, size_t scratch_floats, int* d_err,
                     cudaStream_t s) {
    if (m < 0 || n < 0 || k <= 0 || lda < k || ldb < n || ldc < n)
        return fail(FJ_ERR_SHAPE, "tc_gemm: m=%d n=%d k=%d lda=%d ldb=%d ldc=%d", m, n, k, lda, ldb, ldc);
    if (passes != 1 && passes != 3) return fail(FJ_ERR_SHAPE, "tc_gemm: passes=%d (1 or 3)", passes);
    if (m == 0 || n == 0) return FJ_OK;
    const int kp = (k + kBK - 1) / kBK * kBK;
    const bool split = passes == 3;
    if (scratch == nullptr || scratch_floats < tc_gemm_scratch_floats(m, n, k, passes) ||
        ((uintptr_t)scratch & 15) != 0 || tensor_map_encoder() == nullptr)
        return tc_gemm_tf32(a, lda, b, ldb, c, ldc, m, n, k, alpha, beta, passes, d_err, s);
    float* a_hi = scratch;
    float* a_lo = split ? a_hi + (size_t)m * kp : nullptr;
    float* b_hi = a_hi + (size_t)m * kp * (split ? 2 : 1);
    float* b_lo = split ? b_hi + (size_t)n * kp : nullptr;
    const int64_t ta = (int64_t)m * kp;
    const int row_ctas = (int)std::min<int64_t>((ta + 255) / 256, 148 * 4);
    const int col_ctas = ((n + 31) / 32) * (kp / 32);
    tc_split_kernel<<<(unsigned)(row_ctas + col_ctas), 256, 0, s>>>(a, lda, m, b, ldb, n, k, kp, a_hi, a_lo, b_hi, b_lo,
                                                                   row_ctas);
    note_launch();
    CUtensorMap mah, mal, mbh, mbl;
    // rows are 16-byte multiples (kp x 4 bytes) and every box starts at a multiple of 32 floats
    if (!encode_slabs(&mah, a_hi, m, kp) || !encode_slabs(&mbh, b_hi, n, kp) ||
        !encode_slabs(&mal, split ? a_lo : a_hi, m, kp) || !encode_slabs(&mbl, split ? b_lo : b_hi, n, kp))
        return fail(FJ_ERR_CUDA, "tc_gemm: cuTensorMapEncodeTiled failed");
    FJ_TRY(allow_dynamic_smem((const void*)tc_gemm_tma_kernel, kTmaSmem));
    dim3 grid((unsigned)((n + kBN - 1) / kBN), (unsigned)((m + kBM - 1) / kBM));
    tc_gemm_tma_kernel<<<grid, kTmaThreads, kTmaSmem, s>>>(mah, mal, mbh, mbl, c, ldc, m, n, kp, alpha, beta, passes,
                                                           d_err);
    note_launch();
    FJ_LAUNCH_CHECK("tc_gemm_tma_kernel");
    return FJ_OK;
}

int tri_inverse32_blocks(const float* lu, int n, int b0, int nb, bool upper, float* out, cudaStream_t s) {
    if (n <= 0 || b0 < 0 || nb <= 0 || (b0 + nb - 1) * 128 >= n)
        return fail(FJ_ERR_SHAPE, "tri_inverse: n=%d blocks %d..%d", n, b0, b0 + nb - 1);
    FJ_TRY(allow_dynamic_smem((const void*)tri_inv_kernel, kTriSmem));
    tri_inv_kernel<<<(unsigned)nb, 512, kTriSmem, s>>>(lu, n, b0, upper, out);
    note_launch();
    FJ_LAUNCH_CHECK("tri_inv_kernel");
    return FJ_OK;
}

}  // namespace fj

// Failure-detection self-test: the GEMM kernel with its MMAs and commits withheld, so
// that nothing ever completes the mbarrier it waits on.  Its bounded wait expires (about
// a second), it records the failure, waits (bounded) once more, frees its tensor memory
// and returns; the context stays usable.
extern "C" int fj_tc_wait_selftest(int* d_err, float* d_scratch, fj_stream_t stream) {
    if (!d_err || !d_scratch) return fj::fail(FJ_ERR_SHAPE, "tc_wait_selftest: null pointer");
    float* buf = d_scratch;  // a, b, c of a 1 x 1 x 1 product
    cudaStream_t s = (cudaStream_t)stream;
    FJ_CUDA(cudaMemsetAsync(buf, 0, 4 * sizeof(float), s));
    FJ_TRY(fj::allow_dynamic_smem((const void*)fj::tc_gemm_tf32_kernel, fj::kGemmSmem));
    fj::tc_gemm_tf32_kernel<<<1, fj::kThreads, fj::kGemmSmem, s>>>(buf, 1, buf + 1, 1, buf + 2, 1, 1, 1, 1, 1.0f, 0.0f,
                                                                   0, d_err);
    fj::note_launch();
    FJ_LAUNCH_CHECK("tc_gemm_tf32_kernel (wait self-test)");
    return FJ_OK;
}

extern "C" int fj_gemm_tf32(const float* d_a, int lda, const float* d_b, int ldb, float* d_c, int ldc, int m, int n,
                            int k, float alpha, float beta, int passes, int* d_err, fj_stream_t stream) {
    if (!d_a || !d_b || !d_c || !d_err) return fj::fail(FJ_ERR_SHAPE, "gemm_tf32: null pointer");
    return fj::tc_gemm_tf32(d_a, lda, d_b, ldb, d_c, ldc, m, n, k, alpha, beta, passes, d_err, (cudaStream_t)stream);
}

extern "C" int fj_gemm_tf32_scratch_floats(int m, int n, int k, int passes, size_t* floats) {
    if (!floats || m < 0 || n < 0 || k <= 0 || (passes != 1 && passes != 3))
        return fj::fail(FJ_ERR_SHAPE, "gemm_tf32_scratch_floats: m=%d n=%d k=%d passes=%d", m, n, k, passes);
    *floats = fj::tc_gemm_scratch_floats(m, n, k, passes);
    return FJ_OK;
}

extern "C" int fj_gemm_tf32_tma(const float* d_a, int lda, const float* d_b, int ldb, float* d_c, int ldc, int m,
                                int n, int k, float alpha, float beta, int passes, float* d_scratch,
                                size_t scratch_floats, int* d_err, fj_stream_t stream) {
    if (!d_a || !d_b || !d_c || !d_err || !d_scratch) return fj::fail(FJ_ERR_SHAPE, "gemm_tf32_tma: null pointer");
    if (scratch_floats < fj::tc_gemm_scratch_floats(m, n, k, passes) || ((uintptr_t)d_scratch & 15) != 0)
        return fj::fail(FJ_ERR_SHAPE, "gemm_tf32_tma: scratch of %zu floats at %p (%zu floats, 16-byte aligned)",
                        scratch_floats, (void*)d_scratch, fj::tc_gemm_scratch_floats(m, n, k, passes));
    return fj::tc_gemm_tf32_tma(d_a, lda, d_b, ldb, d_c, ldc, m, n, k, alpha, beta, passes, d_scratch, scratch_floats,
                                d_err, (cudaStream_t)stream);
}
