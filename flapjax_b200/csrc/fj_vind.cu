// fj_vind.cu -- stream packing and the all-pairs Biot-Savart sums (FP64 and FP32).
//
// FP64 path: each (target, filament) pair is evaluated with the reference's own
// formulas (aero/utils.py:580-648) and the products with the filament strengths summed
// in FP64 (aero/aic.py:237-242).
//
// FP32 path ("mixed"): the same sum with
//   - differences x - y formed from hi+lo FP32 splits of the FP64 coordinates,
//   - MUFU rsqrt / fast division,
//   - an explicit collinearity test (sin < kCollinearSin -> exactly 0) standing in for
//     the epsilon regulariser, which FP32 cannot resolve (EPSILON*|r0|^4 ~ 1e-12 is far
//     below FP32 noise in |r1 x r2|^2),
//   - FP32 sums over one staged chunk of filaments, added into FP64 accumulators.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <vector>

#include "fj_bs.cuh"
#include "fj_vind.cuh"

namespace fj {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

const char* last_error() { return g_err; }

static std::atomic<int64_t> g_launches{0};
void note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int allow_dynamic_smem(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    FJ_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    size_t& cur = limit[{dev, func}];
    if (bytes > cur) {
        FJ_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        cur = bytes;
    }
    return FJ_OK;
}
int64_t launch_count() { return g_launches.load(); }

struct ProfState {
    std::mutex mu;
    bool on = false;
    std::vector<cudaEvent_t> ev;  // 2 per slot
    std::vector<double> pairs;
    std::vector<char> fp64;
    int used = 0;
    int64_t launches0 = 0;
};
static ProfState g_prof;
constexpr int kMaxProfSlots = 1 << 16;

int prof_start(cudaStream_t s) {
    std::lock_guard<std::mutex> g(g_prof.mu);
    if (!g_prof.on || g_prof.used >= kMaxProfSlots) return -1;
    const int slot = g_prof.used;
    while ((int)g_prof.ev.size() < 2 * (slot + 1)) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return -1;
        g_prof.ev.push_back(e);
    }
    if ((int)g_prof.pairs.size() <= slot) {
        g_prof.pairs.resize(slot + 1);
        g_prof.fp64.resize(slot + 1);
    }
    cudaEventRecord(g_prof.ev[2 * slot], s);
    g_prof.used = slot + 1;
    return slot;
}

void prof_stop(int slot, cudaStream_t s, double pairs, bool fp64) {
    if (slot < 0) return;
    std::lock_guard<std::mutex> g(g_prof.mu);
    cudaEventRecord(g_prof.ev[2 * slot + 1], s);
    g_prof.pairs[slot] = pairs;
    g_prof.fp64[slot] = fp64;
}

bool prof_active() {
    std::lock_guard<std::mutex> g(g_prof.mu);
    return g_prof.on;
}

int prof_begin() {
    std::lock_guard<std::mutex> g(g_prof.mu);
    g_prof.on = true;
    g_prof.used = 0;
    g_prof.launches0 = launch_count();
    return FJ_OK;
}

int prof_end(fj_profile* out) {
    std::lock_guard<std::mutex> g(g_prof.mu);
    g_prof.on = false;
    fj_profile r;
    memset(&r, 0, sizeof(r));
    r.launches = launch_count() - g_prof.launches0;
    for (int i = 0; i < g_prof.used; ++i) {
        FJ_CUDA(cudaEventSynchronize(g_prof.ev[2 * i + 1]));
        float ms = 0.f;
        FJ_CUDA(cudaEventElapsedTime(&ms, g_prof.ev[2 * i], g_prof.ev[2 * i + 1]));
        r.vind_ms += ms;
        r.vind_ms_max = std::max(r.vind_ms_max, (double)ms);
        r.vind_pairs += g_prof.pairs[i];
        if (g_prof.fp64[i]) {
            r.vind64_launches += 1;
            r.vind64_ms += ms;
            r.vind64_pairs += g_prof.pairs[i];
        }
    }
    r.vind_launches = g_prof.used;
    if (out) *out = r;
    return FJ_OK;
}

// ------------------------------------------------------------------------------------
// Stream packing
// ------------------------------------------------------------------------------------
struct PackedLink {
    double v[3];
    double g;
    double r0[3];
    double q;
};

__device__ __forceinline__ void lattice_vertex(const LatticeRef& L, const MirrorPlane& mp, int k,
                                               int l, double out[3]) {
    const double* p = L.zeta + ((int64_t)k * (L.cols + 1) + l) * 3;
    double z0 = p[0], z1 = p[1], z2 = p[2];
    if (L.mirrored) {
        // mirror_grid, aero/utils.py:651-663
        double d0 = z0 - mp.p[0], d1 = z1 - mp.p[1], d2 = z2 - mp.p[2];
        double dn = d0 * mp.nrm[0] + d1 * mp.nrm[1] + d2 * mp.nrm[2];
        z0 = z0 - 2.0 * dn * mp.nrm[0];
        z1 = z1 - 2.0 * dn * mp.nrm[1];
        z2 = z2 - 2.0 * dn * mp.nrm[2];
    }
    out[0] = z0;
    out[1] = z1;
    out[2] = z2;
}

__device__ __forceinline__ double ring_gamma(const LatticeRef& L, int k, int l) {
    if (k < 0 || l < 0 || k >= L.rows || l >= L.cols) return 0.0;
    return L.gamma[(int64_t)k * L.cols + l];
}

__device__ void pack_one(const PackArgs& a, int64_t e, PackedLink& o) {
    int li = 0;
    while (li + 1 < a.n_lat && e >= a.offset[li + 1]) ++li;
    const LatticeRef& L = a.lat[li];
    int64_t j = e - a.offset[li];
    const int R = L.rows, C = L.cols;
    const int64_t n_chord = (int64_t)(C + 1) * (R + 1);
    int k, l, k1, l1;
    bool brk;
    double g;
    if (j < n_chord) {
        // chordwise chain l: zeta[k,l] -> zeta[k+1,l], strength G[k,l] - G[k,l-1]
        l = (int)(j / (R + 1));
        k = (int)(j % (R + 1));
        brk = (k == R);
        k1 = k + 1;
        l1 = l;
        g = brk ? 0.0 : ring_gamma(L, k, l) - ring_gamma(L, k, l - 1);
    } else {
        // spanwise chain k: zeta[k,l] -> zeta[k,l+1], strength G[k-1,l] - G[k,l]
        int64_t jj = j - n_chord;
        k = (int)(jj / (C + 1));
        l = (int)(jj % (C + 1));
        brk = (l == C);
        k1 = k;
        l1 = l + 1;
        g = brk ? 0.0 : ring_gamma(L, k - 1, l) - ring_gamma(L, k, l);
    }
    lattice_vertex(L, a.mirror, k, l, o.v);
    o.g = g * (double)L.sign;
    if (brk) {
        o.r0[0] = o.r0[1] = o.r0[2] = 0.0;
        o.q = -1.0;
        return;
    }
    double w[3];
    lattice_vertex(L, a.mirror, k1, l1, w);
    o.r0[0] = w[0] - o.v[0];
    o.r0[1] = w[1] - o.v[1];
    o.r0[2] = w[2] - o.v[2];
    const double r0sq = o.r0[0] * o.r0[0] + o.r0[1] * o.r0[1] + o.r0[2] * o.r0[2];
    if (a.kernel == FJ_KERNEL_EPSILON)
        o.q = kEps * r0sq * r0sq;  // aero/utils.py:621-622
    else
        o.q = r0sq;
}

__global__ void pack64_kernel(PackArgs a, Elem64* __restrict__ out) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.offset[a.n_lat]) return;
    PackedLink o;
    pack_one(a, e, o);
    Elem64 r;
    r.x = o.v[0];
    r.y = o.v[1];
    r.z = o.v[2];
    r.g = o.g;
    r.r0x = o.r0[0];
    r.r0y = o.r0[1];
    r.r0z = o.r0[2];
    r.q = o.q;
    out[e] = r;
}

__global__ void pack32_kernel(PackArgs a, Elem32* __restrict__ out) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.offset[a.n_lat]) return;
    PackedLink o;
    pack_one(a, e, o);
    Elem32 r;
    r.xh = (float)o.v[0];
    r.yh = (float)o.v[1];
    r.zh = (float)o.v[2];
    r.xl = (float)(o.v[0] - (double)r.xh);
    r.yl = (float)(o.v[1] - (double)r.yh);
    r.zl = (float)(o.v[2] - (double)r.zh);
    r.g = (float)(o.g / kFourPi);
    r.r0x = (float)o.r0[0];
    r.r0y = (float)o.r0[1];
    r.r0z = (float)o.r0[2];
    if (o.q < 0.0)  // chain break: g = 0 and a q that keeps the link finite (eps) or
        r.q = a.kernel == FJ_KERNEL_EPSILON ? 1.0f : 3.0e38f;  // never kept (cutoff)
    else if (a.kernel == FJ_KERNEL_EPSILON)
        r.q = (float)o.q;
    else  // cutoff: keep iff |r1 x r2|^2 > r_cut^2 |r0|^2  (aero/utils.py:637-648)
        r.q = (float)(a.r_cut * a.r_cut * o.q);
    r.pad = 0.f;
    out[e] = r;
}

__global__ void pack_jobs_kernel(const PackJob* __restrict__ jobs, int fp64) {
    const PackJob& J = jobs[blockIdx.y];
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= J.a.offset[J.a.n_lat]) return;
    PackedLink o;
    pack_one(J.a, e, o);
    if (fp64) {
        Elem64 r;
        r.x = o.v[0];
        r.y = o.v[1];
        r.z = o.v[2];
        r.g = o.g;
        r.r0x = o.r0[0];
        r.r0y = o.r0[1];
        r.r0z = o.r0[2];
        r.q = o.q;
        ((Elem64*)J.out)[e] = r;
    } else {
        Elem32 r;
        r.xh = (float)o.v[0];
        r.yh = (float)o.v[1];
        r.zh = (float)o.v[2];
        r.xl = (float)(o.v[0] - (double)r.xh);
        r.yl = (float)(o.v[1] - (double)r.yh);
        r.zl = (float)(o.v[2] - (double)r.zh);
        r.g = (float)(o.g / kFourPi);
        r.r0x = (float)o.r0[0];
        r.r0y = (float)o.r0[1];
        r.r0z = (float)o.r0[2];
        if (o.q < 0.0)
            r.q = J.a.kernel == FJ_KERNEL_EPSILON ? 1.0f : 3.0e38f;
        else if (J.a.kernel == FJ_KERNEL_EPSILON)
            r.q = (float)o.q;
        else
            r.q = (float)(J.a.r_cut * J.a.r_cut * o.q);
        r.pad = 0.f;
        ((Elem32*)J.out)[e] = r;
    }
}

int pack_jobs(const PackJob* d_jobs, int n_jobs, int64_t max_elem, int precision, cudaStream_t s) {
    if (n_jobs == 0 || max_elem == 0) return FJ_OK;
    dim3 g((unsigned)((max_elem + 255) / 256), (unsigned)n_jobs);
    pack_jobs_kernel<<<g, 256, 0, s>>>(d_jobs, precision == FJ_PREC_FP64); note_launch();
    FJ_LAUNCH_CHECK("pack_jobs_kernel");
    return FJ_OK;
}

int pack_stream64(const PackArgs& a, Elem64* out, cudaStream_t s) {
    int64_t n = a.offset[a.n_lat];
    if (n == 0) return FJ_OK;
    pack64_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, out); note_launch();
    FJ_LAUNCH_CHECK("pack64_kernel");
    return FJ_OK;
}

int pack_stream32(const PackArgs& a, Elem32* out, cudaStream_t s) {
    int64_t n = a.offset[a.n_lat];
    if (n == 0) return FJ_OK;
    pack32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, out); note_launch();
    FJ_LAUNCH_CHECK("pack32_kernel");
    return FJ_OK;
}

// ------------------------------------------------------------------------------------
// FP64 sum: the reference's kernels, evaluated on chains.
// ------------------------------------------------------------------------------------
constexpr int kBlock = 128;  // threads per CTA == staged elements per chunk

template <int KER, int T>
__device__ __forceinline__ void vind64_body(const double* __restrict__ tgt, int64_t n_t,
                                            const Elem64* __restrict__ st, int64_t n_elem, int n_split,
                                            double* __restrict__ part, double rc2, int64_t tile, int split) {
    __shared__ Elem64 sh[kBlock];
    const int64_t per = (n_elem + n_split - 1) / n_split;
    const int64_t e0 = (int64_t)split * per;
    const int64_t e1 = min(n_elem, e0 + per);  // links [e0, e1)
    const int64_t vend = min(e1, n_elem - 1);  // last vertex needed

    double x[T][3];
    int64_t ti[T];
#pragma unroll
    for (int j = 0; j < T; ++j) {
        ti[j] = tile * kBlock * T + threadIdx.x + (int64_t)j * kBlock;
        const int64_t tc = min(ti[j], n_t - 1);
        x[j][0] = tgt[tc * 3 + 0];
        x[j][1] = tgt[tc * 3 + 1];
        x[j][2] = tgt[tc * 3 + 2];
    }
    double acc[T][3];
#pragma unroll
    for (int j = 0; j < T; ++j) acc[j][0] = acc[j][1] = acc[j][2] = 0.0;

    if (e0 < e1) {
        Vtx64<KER> prev[T];
        Elem64 pl = st[e0];
#pragma unroll
        for (int j = 0; j < T; ++j) vtx64<KER>(x[j], pl.x, pl.y, pl.z, prev[j]);
        for (int64_t c0 = e0 + 1; c0 <= vend; c0 += kBlock) {
            const int cnt = (int)min((int64_t)kBlock, vend + 1 - c0);
            __syncthreads();
            if (threadIdx.x < cnt) sh[threadIdx.x] = st[c0 + threadIdx.x];
            __syncthreads();
            for (int i = 0; i < cnt; ++i) {
                const Elem64 cur = sh[i];
#pragma unroll
                for (int j = 0; j < T; ++j) {
                    Vtx64<KER> v;
                    vtx64<KER>(x[j], cur.x, cur.y, cur.z, v);
                    if (pl.q >= 0.0) link64<KER>(prev[j], v, pl.g, pl.r0x, pl.r0y, pl.r0z, pl.q, rc2, acc[j]);
                    prev[j] = v;
                }
                pl = cur;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < T; ++j) {
        if (ti[j] < n_t) {
            double* o = part + ((int64_t)split * n_t + ti[j]) * 3;
            o[0] = acc[j][0];
            o[1] = acc[j][1];
            o[2] = acc[j][2];
        }
    }
}

template <int KER, int T>
__global__ void __launch_bounds__(kBlock) vind64_kernel(VindJob job, double rc2) {
    vind64_body<KER, T>(job.targets, job.n_targets, (const Elem64*)job.stream, job.n_elem, job.n_split, job.part, rc2,
                        blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------------------------------
// FP32 sum.
// ------------------------------------------------------------------------------------
// Packed form: two targets ride in one float2 and every FP32 add/mul/fma of the pair is
// one f32x2 instruction (sm_100: __fadd2_rn / __fmul2_rn / __ffma2_rn), halving the
// issue slots per pair of the scalar form.  The staged element is stored duplicated in
// shared memory ({v, v} pairs, 7 float4), so the broadcast loads give packed operands
// directly.  Subtractions are fma(b, -1, a), which is exact.  T = 2 P targets per thread.
//
// Cancellation-free strength.  The reference's factor r0 . (r1/|r1| - r2/|r2|) subtracts
// two nearly equal unit vectors whenever the target is far from the filament compared with
// its length; in FP32 (and with the approximate MUFU rsqrt) that difference keeps only
// about eps * d / |r0| relative accuracy, so the far field carries an error that decays
// like 1/d instead of 1/d^2 and sums to several 1e-6 of the induced drag.  With
// P = |r1||r2| and D = r1 . r2 the same factor is
//     r0 . (r1/|r1| - r2/|r2|) = (|r1| + |r2|) (P - D) / P,
// and P - D = |r1 x r2|^2 / (P + D).  The kernel takes the second form where D > 0 (the
// far side, where P - D cancels and P + D does not) and the first where D <= 0:
//     epsilon: coef = g S N / (P M (|c|^2 + q)),  N = |c|^2, M = P + D (D > 0); N = P - D, M = 1
//     cutoff:  coef = g S X / (P Y),              X = 1, Y = P + D (D > 0);   X = P - D, Y = |c|^2
// with S = |r1| + |r2|; every term is well conditioned.  The products in the denominators
// are of degree 8 (epsilon) and 4 (cutoff) in the lattice's lengths: FP32 keeps them in
// range for filament lengths and target distances between about 1e-4 and 1e4.
//
// Cross product.  c = r1 x r2 = r0 x r1 (r2 = r1 - r0), formed from the staged filament
// vector r0 and its negation, two instructions per component.  A target on the link's
// start (r1 = 0 exactly, as free-wake vertices are) gives c = 0 exactly; a target on its
// end (r2 = 0 exactly) leaves a rounding residue in r0 x r1, so a vertex whose distance
// is exactly zero carries an infinite collinearity scale s, and the test |c|^2 > s_a s_b
// drops every link that ends there -- the exact zero of the reference's r1 x r2.
struct Vtx32x2 {
    float2 d[3];
    float2 n;  // ||d||_eps
    float2 s;  // kCollinearSin * ||d||_eps^2, or +inf where d = 0
};

// Staged element: vertex part v[0..2] = {hx,hx,hy,hy}, {hz,hz,lx,lx}, {ly,ly,lz,lz}; link
// part l[0..3] = {g,g,q,q}, {r0x,r0x,r0y,r0y}, {r0z,r0z,-r0x,-r0x}, {-r0y,-r0y,-r0z,-r0z}.
constexpr int kDup = 7;  // float4 per staged element
// Six resident CTAs per SM (registers capped at 80): the sum is FMA-pipe bound and the
// extra warps hide the MUFU and FMA latencies better than the registers they cost.
constexpr int kMinCtas32 = 6;
// Four targets per thread (two packed pairs) share each staged element between twice the
// targets at about twice the registers: capped at 128 for four resident CTAs per SM (a
// few FP64 accumulators spill; measured 0.5 % faster than 158 registers and three CTAs).
constexpr int kMinCtas32Wide = 4;
template <int T>
struct MinCtas32 {
    static constexpr int value = T == 2 ? kMinCtas32 : kMinCtas32Wide;
};
constexpr int kFold = 16;  // elements per FP32 partial sum (even: the ping-pong takes pairs)

__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

// MUFU approximations with flush-to-zero (PTX rsqrt.approx.ftz / rcp.approx.ftz): the
// arguments here are never subnormal where the result is kept (||d||_eps^2 >= eps^2;
// a denominator below the collinearity threshold is discarded by the select), so the
// subnormal-input handling of the non-ftz forms is skipped.
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float rcp_ftz(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void vtx32x2(const float2 xh[3], const float2 xl[3], const float4* __restrict__ v,
                                        Vtx32x2& o) {
    const float2 neg1 = dup2(-1.0f);
    const float4 v0 = v[0], v1 = v[1], v2 = v[2];
    const float2 hx = make_float2(v0.x, v0.y), hy = make_float2(v0.z, v0.w), hz = make_float2(v1.x, v1.y);
    const float2 lx = make_float2(v1.z, v1.w), ly = make_float2(v2.x, v2.y), lz = make_float2(v2.z, v2.w);
    o.d[0] = __fadd2_rn(__ffma2_rn(hx, neg1, xh[0]), __ffma2_rn(lx, neg1, xl[0]));
    o.d[1] = __fadd2_rn(__ffma2_rn(hy, neg1, xh[1]), __ffma2_rn(ly, neg1, xl[1]));
    o.d[2] = __fadd2_rn(__ffma2_rn(hz, neg1, xh[2]), __ffma2_rn(lz, neg1, xl[2]));
    constexpr float e2 = (float)(kEps * kEps);
    const float2 n2 = __ffma2_rn(o.d[2], o.d[2], __ffma2_rn(o.d[1], o.d[1], __ffma2_rn(o.d[0], o.d[0], dup2(e2))));
    const float2 inv = make_float2(rsqrt_ftz(n2.x), rsqrt_ftz(n2.y));
    o.n = __fmul2_rn(n2, inv);
    const float2 s = __fmul2_rn(n2, dup2(kCollinearSin));
    o.s = make_float2(n2.x > e2 ? s.x : __int_as_float(0x7f800000), n2.y > e2 ? s.y : __int_as_float(0x7f800000));
}

// The link from vertex a (element e) to vertex b (element e+1) with element e's link part l.
template <int KER>
__device__ __forceinline__ void link32x2(const Vtx32x2& a, const Vtx32x2& b, const float4* __restrict__ l,
                                         float2 acc[3]) {
    const float2 neg1 = dup2(-1.0f);
    const float4 l0 = l[0], l1 = l[1], l2 = l[2], l3 = l[3];
    const float2 g = make_float2(l0.x, l0.y), q = make_float2(l0.z, l0.w);
    const float2 r0x = make_float2(l1.x, l1.y), r0y = make_float2(l1.z, l1.w), r0z = make_float2(l2.x, l2.y);
    const float2 nx = make_float2(l2.z, l2.w), ny = make_float2(l3.x, l3.y), nz = make_float2(l3.z, l3.w);
    const float2 cx = __ffma2_rn(r0y, a.d[2], __fmul2_rn(nz, a.d[1]));
    const float2 cy = __ffma2_rn(r0z, a.d[0], __fmul2_rn(nx, a.d[2]));
    const float2 cz = __ffma2_rn(r0x, a.d[1], __fmul2_rn(ny, a.d[0]));
    const float2 c2 = __ffma2_rn(cz, cz, __ffma2_rn(cy, cy, __fmul2_rn(cx, cx)));
    const float2 D = __ffma2_rn(a.d[2], b.d[2], __ffma2_rn(a.d[1], b.d[1], __fmul2_rn(a.d[0], b.d[0])));
    const float2 P = __fmul2_rn(a.n, b.n);
    const float2 PpD = __fadd2_rn(P, D);
    const float2 PmD = __ffma2_rn(D, neg1, P);
    const float2 t = __fmul2_rn(a.s, b.s);
    const float2 gS = __fmul2_rn(g, __fadd2_rn(a.n, b.n));
    float2 coef;
    if (KER == FJ_KERNEL_EPSILON) {
        const float2 N = make_float2(D.x > 0.0f ? c2.x : PmD.x, D.y > 0.0f ? c2.y : PmD.y);
        const float2 M = make_float2(D.x > 0.0f ? PpD.x : 1.0f, D.y > 0.0f ? PpD.y : 1.0f);
        const float2 den = __fmul2_rn(__fmul2_rn(P, M), __fadd2_rn(c2, q));
        coef = __fmul2_rn(__fmul2_rn(gS, N), make_float2(rcp_ftz(den.x), rcp_ftz(den.y)));
        coef.x = c2.x > t.x ? coef.x : 0.0f;
        coef.y = c2.y > t.y ? coef.y : 0.0f;
    } else {
        const float2 X = make_float2(D.x > 0.0f ? 1.0f : PmD.x, D.y > 0.0f ? 1.0f : PmD.y);
        const float2 Y = make_float2(D.x > 0.0f ? PpD.x : c2.x, D.y > 0.0f ? PpD.y : c2.y);
        const float2 den = __fmul2_rn(P, Y);
        coef = __fmul2_rn(__fmul2_rn(gS, X), make_float2(rcp_ftz(den.x), rcp_ftz(den.y)));
        coef.x = c2.x > fmaxf(q.x, t.x) ? coef.x : 0.0f;
        coef.y = c2.y > fmaxf(q.y, t.y) ? coef.y : 0.0f;
    }
    acc[0] = __ffma2_rn(cx, coef, acc[0]);
    acc[1] = __ffma2_rn(cy, coef, acc[1]);
    acc[2] = __ffma2_rn(cz, coef, acc[2]);
}

__device__ __forceinline__ void stage_dup(const float4* __restrict__ s4, int64_t e, float4* __restrict__ o) {
    const float4 a = s4[e * 3 + 0], b = s4[e * 3 + 1], c = s4[e * 3 + 2];  // {xh,yh,zh,g} {xl,yl,zl,q} {r0,pad}
    o[0] = make_float4(a.x, a.x, a.y, a.y);
    o[1] = make_float4(a.z, a.z, b.x, b.x);
    o[2] = make_float4(b.y, b.y, b.z, b.z);
    o[3] = make_float4(a.w, a.w, b.w, b.w);
    o[4] = make_float4(c.x, c.x, c.y, c.y);
    o[5] = make_float4(c.z, c.z, -c.x, -c.x);
    o[6] = make_float4(-c.y, -c.y, -c.z, -c.z);
}

template <int KER, int T>
__device__ __forceinline__ void vind32_body(const double* __restrict__ tgt, int64_t n_t,
                                            const Elem32* __restrict__ st, int64_t n_elem, int n_split,
                                            double* __restrict__ part, int64_t tile, int split) {
    static_assert(T % 2 == 0, "targets come in pairs");
    constexpr int P = T / 2;
    // slot 0: the element before the chunk (owner of the chunk's first link); 1..cnt: chunk
    __shared__ float4 sh[(kBlock + 1) * kDup];
    const int64_t per = (n_elem + n_split - 1) / n_split;
    const int64_t e0 = (int64_t)split * per;
    const int64_t e1 = min(n_elem, e0 + per);
    const int64_t vend = min(e1, n_elem - 1);

    // pack p holds targets j = 2p (.x) and 2p+1 (.y); target j is threadIdx.x + j kBlock
    float2 xh[P][3], xl[P][3];
    int64_t ti[T];
#pragma unroll
    for (int j = 0; j < T; ++j) ti[j] = tile * kBlock * T + threadIdx.x + (int64_t)j * kBlock;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int64_t ta = min(ti[2 * p], n_t - 1), tb = min(ti[2 * p + 1], n_t - 1);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double va = tgt[ta * 3 + c], vb = tgt[tb * 3 + c];
            xh[p][c] = make_float2((float)va, (float)vb);
            xl[p][c] = make_float2((float)(va - (double)xh[p][c].x), (float)(vb - (double)xh[p][c].y));
        }
    }
    double acc[T][3];
#pragma unroll
    for (int j = 0; j < T; ++j) acc[j][0] = acc[j][1] = acc[j][2] = 0.0;

    if (e0 < e1) {
        const float4* s4 = reinterpret_cast<const float4*>(st);
        // A: vertex of the element owning the next link; B: the one after (ping-pong)
        Vtx32x2 A[P], B[P];
        {
            float4 first[kDup];
            stage_dup(s4, e0, first);
#pragma unroll
            for (int p = 0; p < P; ++p) vtx32x2(xh[p], xl[p], first, A[p]);
        }
        for (int64_t c0 = e0 + 1; c0 <= vend; c0 += kBlock) {
            const int cnt = (int)min((int64_t)kBlock, vend + 1 - c0);
            __syncthreads();
            for (int k = threadIdx.x; k <= cnt; k += kBlock) stage_dup(s4, c0 - 1 + k, sh + k * kDup);
            __syncthreads();
            // FP32 partial sums over kFold elements, folded into the FP64 accumulators:
            // bounds the FP32 summation error to that of a 16-term sum
            for (int f0 = 0; f0 < cnt; f0 += kFold) {
                const int fend = min(cnt, f0 + kFold);
                float2 accf[P][3];
#pragma unroll
                for (int p = 0; p < P; ++p) accf[p][0] = accf[p][1] = accf[p][2] = make_float2(0.f, 0.f);
                // Chain breaks carry g = 0 and a q that keeps their (discarded) term
                // finite, so every element is processed without a branch.
                int i = f0;
                for (; i + 2 <= fend; i += 2) {
                    const float4* e = sh + i * kDup;  // slots i, i+1, i+2
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        vtx32x2(xh[p], xl[p], e + kDup, B[p]);
                        link32x2<KER>(A[p], B[p], e + 3, accf[p]);
                    }
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        vtx32x2(xh[p], xl[p], e + 2 * kDup, A[p]);
                        link32x2<KER>(B[p], A[p], e + kDup + 3, accf[p]);
                    }
                }
                if (i < fend) {
                    const float4* e = sh + i * kDup;
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        vtx32x2(xh[p], xl[p], e + kDup, B[p]);
                        link32x2<KER>(A[p], B[p], e + 3, accf[p]);
                        A[p] = B[p];
                    }
                }
#pragma unroll
                for (int p = 0; p < P; ++p)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        acc[2 * p][c] += (double)accf[p][c].x;
                        acc[2 * p + 1][c] += (double)accf[p][c].y;
                    }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < T; ++j) {
        if (ti[j] < n_t) {
            double* o = part + ((int64_t)split * n_t + ti[j]) * 3;
            o[0] = acc[j][0];
            o[1] = acc[j][1];
            o[2] = acc[j][2];
        }
    }
}

template <int KER, int T>
__global__ void __launch_bounds__(kBlock, MinCtas32<T>::value) vind32_kernel(VindJob job) {
    vind32_body<KER, T>(job.targets, job.n_targets, (const Elem32*)job.stream, job.n_elem, job.n_split, job.part,
                        blockIdx.x, blockIdx.y);
}

// Many jobs in one launch: CTA b belongs to the job j with cta0[j] <= b < cta0[j+1];
// within a job, CTAs are numbered tile-fastest (tile + ctas_x * split).
__device__ __forceinline__ int find_job(const int64_t* __restrict__ cta0, int n_jobs, int64_t b) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cta0[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The grid walks the virtual CTAs 0 .. cta0[n_jobs]-1 of the job table in strides of its
// size.  Launched with one CTA per virtual CTA it is the plain tiled sum; launched
// persistent (a fixed grid: the CTAs the GPU holds at once) the launch does not depend on
// the jobs' sizes, so one captured launch serves any batch of the same job count.  The
// persistent form is not the default: its last round of virtual CTAs can fall on a subset
// of the SMs (9 % slower on the 16 x 128 free-wake step than hardware scheduling, whose
// last partial wave spreads over every SM).
template <int KER, int T>
__global__ void __launch_bounds__(kBlock, MinCtas32<T>::value) vind32_jobs_kernel(const VindJob* __restrict__ jobs,
                                                             const int64_t* __restrict__ cta0, int n_jobs) {
    const int64_t total = cta0[n_jobs];
    for (int64_t b = blockIdx.x; b < total; b += gridDim.x) {
        const int j = find_job(cta0, n_jobs, b);
        const VindJob job = jobs[j];
        const int64_t local = b - cta0[j];
        const int64_t ctas_x = (job.n_targets + (int64_t)kBlock * T - 1) / ((int64_t)kBlock * T);
        vind32_body<KER, T>(job.targets, job.n_targets, (const Elem32*)job.stream, job.n_elem, job.n_split, job.part,
                            local % ctas_x, (int)(local / ctas_x));
    }
}

template <int KER, int T>
__global__ void __launch_bounds__(kBlock) vind64_jobs_kernel(const VindJob* __restrict__ jobs,
                                                             const int64_t* __restrict__ cta0, int n_jobs,
                                                             double rc2) {
    const int64_t total = cta0[n_jobs];
    for (int64_t b = blockIdx.x; b < total; b += gridDim.x) {
        const int j = find_job(cta0, n_jobs, b);
        const VindJob job = jobs[j];
        const int64_t local = b - cta0[j];
        const int64_t ctas_x = (job.n_targets + (int64_t)kBlock * T - 1) / ((int64_t)kBlock * T);
        vind64_body<KER, T>(job.targets, job.n_targets, (const Elem64*)job.stream, job.n_elem, job.n_split, job.part,
                            rc2, local % ctas_x, (int)(local / ctas_x));
    }
}

__global__ void reduce_partials_kernel(const double* __restrict__ part, int n_split, int64_t n3,
                                       double* __restrict__ out, int accumulate, double scale) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    double s = 0.0;
    for (int k = 0; k < n_split; ++k) s += part[(int64_t)k * n3 + i];
    s *= scale;
    out[i] = accumulate ? out[i] + s : s;
}

__global__ void reduce_jobs_kernel(const VindJob* __restrict__ jobs) {
    const VindJob& J = jobs[blockIdx.y];
    const int64_t n3 = J.n_targets * 3;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    double sacc = 0.0;
    for (int k = 0; k < J.n_split; ++k) sacc += J.part[(int64_t)k * n3 + i];
    J.out[i] = J.accumulate ? J.out[i] + sacc : sacc;
}

int reduce_jobs(const VindJob* d_jobs, int n_jobs, int64_t max_targets, cudaStream_t s) {
    if (n_jobs == 0 || max_targets == 0) return FJ_OK;
    dim3 g((unsigned)((max_targets * 3 + 255) / 256), (unsigned)n_jobs);
    reduce_jobs_kernel<<<g, 256, 0, s>>>(d_jobs); note_launch();
    FJ_LAUNCH_CHECK("reduce_jobs_kernel");
    return FJ_OK;
}

int reduce_partials(const double* part, int n_split, int64_t n_targets, double* out, int accumulate,
                    double scale, cudaStream_t s) {
    const int64_t n3 = n_targets * 3;
    if (n3 == 0) return FJ_OK;
    reduce_partials_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(part, n_split, n3, out,
                                                                         accumulate, scale); note_launch();
    FJ_LAUNCH_CHECK("reduce_partials_kernel");
    return FJ_OK;
}

constexpr int kT64 = 2;
constexpr int kT32 = 2;      // FP32 targets per thread unless the tuned table says otherwise
constexpr int kT32Wide = 4;  // the wide tile the autotuner may choose instead
constexpr int kTileWideFlag = 0x1000;  // tuned entry: split | flag when the wide tile won

// CTAs resident per SM for the sum kernels and the SM count, queried once.
static int g_sms = 0, g_res64 = 0, g_res32 = 0, g_res32w = 0;

static std::once_flag g_occ_once;

static void query_occupancy() {
    std::call_once(g_occ_once, [] {
        int dev = 0;
        cudaGetDevice(&dev);
        int sms = 0, r64 = 0, r32 = 0, r32w = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r64, vind64_kernel<FJ_KERNEL_EPSILON, kT64>, kBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r32, vind32_kernel<FJ_KERNEL_CUTOFF, kT32>, kBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r32w, vind32_kernel<FJ_KERNEL_CUTOFF, kT32Wide>, kBlock, 0);
        g_res64 = r64 > 0 ? r64 : 1;
        g_res32 = r32 > 0 ? r32 : 1;
        g_res32w = r32w > 0 ? r32w : 1;
        g_sms = sms > 0 ? sms : 148;
    });
}

// Split the stream so that (target blocks) x (splits) fills whole waves: the smallest
// split count with at least two waves' worth of CTAs whose last wave is >= 90 % full
// (or the best efficiency found), bounded by >= 256 elements per split.
// Upper bound on choose_split for any stream of at most n_elem_max elements (workspace
// sizing): independent of the device queried.
int split_bound(int64_t n_targets, int64_t n_elem_max, int precision) {
    const int T = precision == FJ_PREC_FP64 ? kT64 : kT32;
    const int64_t ctas = std::max<int64_t>(1, (n_targets + (int64_t)kBlock * T - 1) / ((int64_t)kBlock * T));
    const int64_t cap = (4ll * 160 * 16 + ctas - 1) / ctas;  // 4 waves of 160 SMs x 16 CTAs
    return (int)std::max<int64_t>(1, std::min<int64_t>({1024, cap, std::max<int64_t>(1, n_elem_max / 256)}));
}

// Autotuned splits (fj_autotune_vind): published once per tuning as a whole new table,
// never modified after publication; choose_split reads it lock-free.
static std::atomic<const TuneTable*> g_tune{nullptr};

const TuneTable* tune_table() { return g_tune.load(std::memory_order_acquire); }

void tune_publish(const TuneTable* t) { g_tune.store(t, std::memory_order_release); }

int tune_bucket_targets(int64_t n_targets) {
    int b = 0;
    while (b + 1 < kTuneTargetBuckets && (1ll << (b + 1)) <= n_targets) ++b;
    return b;
}

int tune_bucket_elem(int64_t n_elem) {
    int b = 0;
    while (b + 1 < kTuneElemBuckets && (1ll << (b + 1)) <= n_elem) ++b;
    return b;
}

int choose_split(int64_t n_targets, int64_t n_elem, int precision) {
    if (const TuneTable* t = tune_table()) {
        const int v = t->split[precision == FJ_PREC_FP64 ? 0 : 1][tune_bucket_targets(n_targets)][tune_bucket_elem(n_elem)];
        if (v > 0) return std::min(v & (kTileWideFlag - 1), split_bound(n_targets, n_elem, precision));
    }
    return heuristic_split(n_targets, n_elem, precision);
}

int choose_tile(int64_t n_targets, int64_t n_elem, int precision) {
    if (precision == FJ_PREC_FP64) return kT64;
    if (const TuneTable* t = tune_table()) {
        const int v = t->split[1][tune_bucket_targets(n_targets)][tune_bucket_elem(n_elem)];
        if (v > 0 && (v & kTileWideFlag)) return kT32Wide;
    }
    return kT32;
}

int encode_tuned(int split, int tile) { return split | (tile == kT32Wide ? kTileWideFlag : 0); }

int heuristic_split(int64_t n_targets, int64_t n_elem, int precision) {
    query_occupancy();
    const int T = precision == FJ_PREC_FP64 ? kT64 : kT32;
    const int64_t ctas = (n_targets + (int64_t)kBlock * T - 1) / ((int64_t)kBlock * T);
    int sms = 148, res = precision == FJ_PREC_FP64 ? 4 : 6;
    if (g_sms > 0) {
        sms = g_sms;
        res = precision == FJ_PREC_FP64 ? g_res64 : g_res32;
    }
    const int64_t wave = (int64_t)sms * res;
    const int64_t max_sp = split_bound(n_targets, n_elem, precision);
    int64_t best = 1;
    double best_eff = -1.0;
    for (int64_t sp = 1; sp <= max_sp; ++sp) {
        const int64_t total = ctas * sp;
        const int64_t waves = (total + wave - 1) / wave;
        const double eff = (double)total / (double)(waves * wave);
        if (total >= 2 * wave && eff >= 0.9) return (int)sp;
        if (eff > best_eff + 1e-9 || (total < 2 * wave && eff >= best_eff - 1e-9)) {
            best_eff = eff;
            best = sp;
        }
    }
    return (int)best;
}

int vind_launch(const VindJob& job, int precision, int kernel, double r_cut, cudaStream_t s, int tile) {
    if (job.n_targets == 0) return FJ_OK;
    query_occupancy();
    const int T = precision == FJ_PREC_FP64 ? kT64 : (tile ? tile : choose_tile(job.n_targets, job.n_elem, precision));
    if (T != kT32 && T != kT32Wide) return fail(FJ_ERR_SHAPE, "vind: tile %d (2 or 4 targets per thread)", T);
    const int64_t gx = (job.n_targets + (int64_t)kBlock * T - 1) / ((int64_t)kBlock * T);
    if (gx > 0x7fffffff || job.n_split > 65535) return fail(FJ_ERR_SHAPE, "vind: grid too large");
    dim3 grid((unsigned)gx, (unsigned)job.n_split);
    const int prof = prof_start(s);
    if (precision == FJ_PREC_FP64) {
        const double rc2 = r_cut * r_cut;
        switch (kernel) {
            case FJ_KERNEL_EPSILON:
                vind64_kernel<FJ_KERNEL_EPSILON, kT64><<<grid, kBlock, 0, s>>>(job, rc2); note_launch();
                break;
            case FJ_KERNEL_CUTOFF:
                vind64_kernel<FJ_KERNEL_CUTOFF, kT64><<<grid, kBlock, 0, s>>>(job, rc2); note_launch();
                break;
            case FJ_KERNEL_PLAIN:
                vind64_kernel<FJ_KERNEL_PLAIN, kT64><<<grid, kBlock, 0, s>>>(job, rc2); note_launch();
                break;
            default:
                return fail(FJ_ERR_UNSUPPORTED, "vind: unknown kernel %d", kernel);
        }
    } else {
        switch (kernel) {
            case FJ_KERNEL_EPSILON:
                if (T == kT32) vind32_kernel<FJ_KERNEL_EPSILON, kT32><<<grid, kBlock, 0, s>>>(job);
                else vind32_kernel<FJ_KERNEL_EPSILON, kT32Wide><<<grid, kBlock, 0, s>>>(job);
                note_launch();
                break;
            case FJ_KERNEL_CUTOFF:
                if (T == kT32) vind32_kernel<FJ_KERNEL_CUTOFF, kT32><<<grid, kBlock, 0, s>>>(job);
                else vind32_kernel<FJ_KERNEL_CUTOFF, kT32Wide><<<grid, kBlock, 0, s>>>(job);
                note_launch();
                break;
            default:
                return fail(FJ_ERR_UNSUPPORTED, "vind: kernel %d has no FP32 variant (use FJ_PREC_FP64)", kernel);
        }
    }
    prof_stop(prof, s, (double)job.n_targets * (double)job.n_links, precision == FJ_PREC_FP64);
    FJ_LAUNCH_CHECK("vind kernel");
    return FJ_OK;
}

int64_t vind_ctas(int64_t n_targets, int n_split, int precision, int tile) {
    const int T = precision == FJ_PREC_FP64 ? kT64 : (tile ? tile : kT32);
    return (n_targets + (int64_t)kBlock * T - 1) / ((int64_t)kBlock * T) * n_split;
}

int vind_launch_jobs(const VindJob* d_jobs, const int64_t* d_cta0, int n_jobs, int64_t total_ctas, double pairs,
                     int precision, int kernel, double r_cut, cudaStream_t s, bool persistent, int tile) {
    if (n_jobs == 0 || total_ctas == 0) return FJ_OK;
    if (total_ctas > 0x7fffffff) return fail(FJ_ERR_SHAPE, "vind jobs: grid too large");
    query_occupancy();
    // one CTA per virtual CTA (the hardware schedules them, and a last partial wave spreads
    // over every SM), or, persistent, the CTAs the GPU holds at once whatever the jobs need
    const bool wide = precision != FJ_PREC_FP64 && tile == kT32Wide;
    if (precision != FJ_PREC_FP64 && tile != 0 && tile != kT32 && tile != kT32Wide)
        return fail(FJ_ERR_SHAPE, "vind jobs: tile %d (2 or 4 targets per thread)", tile);
    const int64_t resident = (int64_t)g_sms * (precision == FJ_PREC_FP64 ? g_res64 : (wide ? g_res32w : g_res32));
    const unsigned g = (unsigned)std::max<int64_t>(1, persistent ? resident : total_ctas);
    const int prof = prof_start(s);
    if (precision == FJ_PREC_FP64) {
        const double rc2 = r_cut * r_cut;
        switch (kernel) {
            case FJ_KERNEL_EPSILON:
                vind64_jobs_kernel<FJ_KERNEL_EPSILON, kT64><<<g, kBlock, 0, s>>>(d_jobs, d_cta0, n_jobs, rc2); note_launch();
                break;
            case FJ_KERNEL_CUTOFF:
                vind64_jobs_kernel<FJ_KERNEL_CUTOFF, kT64><<<g, kBlock, 0, s>>>(d_jobs, d_cta0, n_jobs, rc2); note_launch();
                break;
            case FJ_KERNEL_PLAIN:
                vind64_jobs_kernel<FJ_KERNEL_PLAIN, kT64><<<g, kBlock, 0, s>>>(d_jobs, d_cta0, n_jobs, rc2); note_launch();
                break;
            default:
                return fail(FJ_ERR_UNSUPPORTED, "vind: unknown kernel %d", kernel);
        }
    } else {
        switch (kernel) {
            case FJ_KERNEL_EPSILON:
                if (!wide) vind32_jobs_kernel<FJ_KERNEL_EPSILON, kT32><<<g, kBlock, 0, s>>>(d_jobs, d_cta0, n_jobs);
                else vind32_jobs_kernel<FJ_KERNEL_EPSILON, kT32Wide><<<g, kBlock, 0, s>>>(d_jobs, d_cta0, n_jobs);
                note_launch();
                break;
            case FJ_KERNEL_CUTOFF:
                if (!wide) vind32_jobs_kernel<FJ_KERNEL_CUTOFF, kT32><<<g, kBlock, 0, s>>>(d_jobs, d_cta0, n_jobs);
                else vind32_jobs_kernel<FJ_KERNEL_CUTOFF, kT32Wide><<<g, kBlock, 0, s>>>(d_jobs, d_cta0, n_jobs);
                note_launch();
                break;
            default:
                return fail(FJ_ERR_UNSUPPORTED, "vind: kernel %d has no FP32 variant (use FJ_PREC_FP64)", kernel);
        }
    }
    prof_stop(prof, s, pairs, precision == FJ_PREC_FP64);
    FJ_LAUNCH_CHECK("vind jobs kernel");
    return FJ_OK;
}

// ------------------------------------------------------------------------------------
// Pairwise kernel evaluation (the reference's per-pair functions, for known-answer tests)
// ------------------------------------------------------------------------------------
__global__ void bs_pairs_kernel(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                                int kernel, double rc2, double* __restrict__ out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xx[3] = {x[i * 3], x[i * 3 + 1], x[i * 3 + 2]};
    const double* yy = y + i * 6;
    const double r0x = yy[3] - yy[0], r0y = yy[4] - yy[1], r0z = yy[5] - yy[2];
    const double r0sq = r0x * r0x + r0y * r0y + r0z * r0z;
    double acc[3] = {0.0, 0.0, 0.0};
    if (kernel == FJ_KERNEL_EPSILON) {
        Vtx64<FJ_KERNEL_EPSILON> a, b;
        vtx64<FJ_KERNEL_EPSILON>(xx, yy[0], yy[1], yy[2], a);
        vtx64<FJ_KERNEL_EPSILON>(xx, yy[3], yy[4], yy[5], b);
        link64<FJ_KERNEL_EPSILON>(a, b, 1.0, r0x, r0y, r0z, kEps * r0sq * r0sq, rc2, acc);
    } else if (kernel == FJ_KERNEL_CUTOFF) {
        Vtx64<FJ_KERNEL_CUTOFF> a, b;
        vtx64<FJ_KERNEL_CUTOFF>(xx, yy[0], yy[1], yy[2], a);
        vtx64<FJ_KERNEL_CUTOFF>(xx, yy[3], yy[4], yy[5], b);
        link64<FJ_KERNEL_CUTOFF>(a, b, 1.0, r0x, r0y, r0z, r0sq, rc2, acc);
    } else {
        Vtx64<FJ_KERNEL_PLAIN> a, b;
        vtx64<FJ_KERNEL_PLAIN>(xx, yy[0], yy[1], yy[2], a);
        vtx64<FJ_KERNEL_PLAIN>(xx, yy[3], yy[4], yy[5], b);
        link64<FJ_KERNEL_PLAIN>(a, b, 1.0, r0x, r0y, r0z, r0sq, rc2, acc);
    }
    out[i * 3 + 0] = acc[0];
    out[i * 3 + 1] = acc[1];
    out[i * 3 + 2] = acc[2];
}

int biot_savart_pairs(const double* x, const double* y, int64_t n, int kernel, double r_cut,
                      double* out, cudaStream_t s) {
    if (n < 0) return fail(FJ_ERR_SHAPE, "fj_biot_savart: n_pairs < 0");
    if (kernel < 0 || kernel > 2) return fail(FJ_ERR_UNSUPPORTED, "fj_biot_savart: kernel %d", kernel);
    if (n == 0) return FJ_OK;
    bs_pairs_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, y, n, kernel, r_cut * r_cut, out); note_launch();
    FJ_LAUNCH_CHECK("bs_pairs_kernel");
    return FJ_OK;
}

}  // namespace fj

namespace fj {
// Eight independent FMA chains per thread, all in registers.
__global__ void __launch_bounds__(256) fma_peak_kernel(float* out, int iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
    }
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) sum += x[k];
    if (sum == 1234.5f) out[0] = sum;  // keeps the chains live; practically never true
}

// The same with packed f32x2 FMAs (the form the FP32 Biot-Savart sum issues).
__global__ void __launch_bounds__(256) fma2_peak_kernel(float* out, int iters, float a, float b) {
    float2 x[8];
    const float2 A = make_float2(a, a), B = make_float2(b, b);
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = make_float2(threadIdx.x * 1e-3f + k, 0.5f * k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = __ffma2_rn(x[k], A, B);
    }
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) sum += x[k].x + x[k].y;
    if (sum == 1234.5f) out[0] = sum;
}

// FP32 CUDA-core peak (TFLOP/s, FMA = 2): the larger of the scalar and packed FMA-chain
// rates over 8 CTAs of 256 threads per SM, second of two timed launches each.
int peak_fp32(double* tflops, cudaStream_t s) {
    int dev = 0, sms = 0;
    FJ_CUDA(cudaGetDevice(&dev));
    FJ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t e0, e1;
    FJ_CUDA(cudaEventCreate(&e0));
    FJ_CUDA(cudaEventCreate(&e1));
    double best = 0.0;
    for (int packed = 0; packed < 2; ++packed) {
        float ms = 0.f;
        for (int rep = 0; rep < 2; ++rep) {
            cudaEventRecord(e0, s);
            if (packed) {
                fma2_peak_kernel<<<blocks, threads, 0, s>>>(nullptr, iters, 0.999999f, 1e-7f); note_launch();
            } else {
                fma_peak_kernel<<<blocks, threads, 0, s>>>(nullptr, iters, 0.999999f, 1e-7f); note_launch();
            }
            cudaEventRecord(e1, s);
        }
        FJ_LAUNCH_CHECK("fma_peak_kernel");
        FJ_CUDA(cudaEventSynchronize(e1));
        FJ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const double flops = 2.0 * 8.0 * iters * (double)blocks * threads * (packed ? 2.0 : 1.0);
        best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *tflops = best;
    return FJ_OK;
}
}  // namespace fj

extern "C" {
int fj_peak_fp32(double* tflops, fj_stream_t stream) { return fj::peak_fp32(tflops, (cudaStream_t)stream); }
int fj_profile_begin(void) { return fj::prof_begin(); }
int fj_profile_end(fj_profile* out) { return fj::prof_end(out); }
int64_t fj_launch_count(void) { return fj::launch_count(); }
}
