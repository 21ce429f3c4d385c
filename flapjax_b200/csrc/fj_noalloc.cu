// fj_noalloc.cu -- compute_v_ind for callers that cannot allocate device memory.
//
// fj_vind needs scratch memory (the packed filament stream and per-split partial
// velocities), which its caller allocates and passes in.  Some callers cannot do that:
// a plugin host that owns the whole device memory pool and forbids other allocations, or
// a real-time loop that must never block in cudaMalloc.  fj_vind_noalloc serves them with
// scratch that lives in a file-scope __device__ array of fixed size (kNoAllocScratchBytes,
// 8 MiB), reserved on every GPU that loads this library until the process exits.
//
// Host code cannot use the array's name as a device address (on the host it names a
// stand-in object), so the address is fetched with cudaGetSymbolAddress, once per device,
// with that device current, on the first call made on that device.  The fetched address
// is kept for the life of the process: it does not survive cudaDeviceReset (which
// reloads this module), so a caller that resets a device must not call this entry point
// on that device afterwards.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "fj_vind.cuh"

namespace fj {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (set up on first use).
static int noalloc_scratch(char** out) {
    int dev = -1;
    FJ_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return fail(FJ_ERR_UNSUPPORTED, "fj_vind_noalloc: device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(FJ_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    *out = static_cast<char*>(g_noalloc_addr[dev]);
    return FJ_OK;
}

}  // namespace fj

using namespace fj;

extern "C" FJ_API int fj_vind_noalloc(const double* d_targets, int64_t n_targets, const double* const* d_zetas,
                                      const double* const* d_gammas, const int* rows, const int* cols,
                                      int n_lattices, const double* mirror_point, const double* mirror_normal,
                                      int kernel, double r_cut, int precision, double* d_v_out,
                                      fj_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (n_targets < 0 || n_lattices < 0 || n_lattices > FJ_MAX_SURF * 2)
        return fail(FJ_ERR_SHAPE, "fj_vind_noalloc: n_targets=%lld n_lattices=%d", (long long)n_targets, n_lattices);
    if (precision != FJ_PREC_FP64 && precision != FJ_PREC_MIXED)
        return fail(FJ_ERR_UNSUPPORTED, "fj_vind_noalloc: precision %d", precision);
    if (kernel < 0 || kernel > 2) return fail(FJ_ERR_UNSUPPORTED, "fj_vind_noalloc: kernel %d", kernel);
    if (precision == FJ_PREC_MIXED && kernel == FJ_KERNEL_PLAIN)
        return fail(FJ_ERR_UNSUPPORTED, "fj_vind_noalloc: the unregularised kernel is FP64-only");
    const int mirror = mirror_point != nullptr && mirror_normal != nullptr;
    const int img = mirror ? 2 : 1;
    int64_t n_elem = 0, n_links = 0;
    for (int i = 0; i < n_lattices; ++i) {
        if (rows[i] < 0 || cols[i] < 0 || rows[i] >= (1 << 24) || cols[i] >= (1 << 24))
            return fail(FJ_ERR_SHAPE, "fj_vind_noalloc: lattice %d has rows=%d cols=%d", i, rows[i], cols[i]);
        n_elem += img * stream_len(rows[i], cols[i]);
        n_links += img * lattice_links(rows[i], cols[i]);
    }
    // scratch = [stream][partials]; refuse sizes the fixed array cannot hold (the target
    // count first, so that the byte counts below cannot wrap)
    if (n_targets > (int64_t)(kNoAllocScratchBytes / (3 * sizeof(double))) ||
        n_elem > (int64_t)(kNoAllocScratchBytes / sizeof(Elem32)))
        return fail(FJ_ERR_SHAPE,
                    "fj_vind_noalloc: %lld targets and %lld filament-stream elements exceed its fixed %zu-byte "
                    "array; use fj_vind with a caller workspace",
                    (long long)n_targets, (long long)n_elem, kNoAllocScratchBytes);
    const size_t elem_bytes = precision == FJ_PREC_FP64 ? sizeof(Elem64) : sizeof(Elem32);
    const size_t stream_bytes = align_up((size_t)n_elem * elem_bytes, 256);
    const size_t part_per_split = (size_t)std::max<int64_t>(n_targets, 1) * 3 * sizeof(double);
    if (stream_bytes + part_per_split > kNoAllocScratchBytes)
        return fail(FJ_ERR_SHAPE,
                    "fj_vind_noalloc: %lld filament-stream elements and %lld targets need %zu bytes of scratch, "
                    "more than its fixed %zu-byte array; use fj_vind with a caller workspace",
                    (long long)n_elem, (long long)n_targets, stream_bytes + part_per_split, kNoAllocScratchBytes);
    if (n_targets == 0) return FJ_OK;

    char* scratch = nullptr;
    FJ_TRY(noalloc_scratch(&scratch));
    if (n_elem == 0) return cuda_status(cudaMemsetAsync(d_v_out, 0, n_targets * 3 * sizeof(double), s), "memset");

    PackArgs pa;
    memset(&pa, 0, sizeof(pa));
    pa.kernel = kernel;
    pa.r_cut = r_cut;
    if (mirror)
        for (int d = 0; d < 3; ++d) {
            pa.mirror.p[d] = mirror_point[d];
            pa.mirror.nrm[d] = mirror_normal[d];
        }
    int n = 0;
    for (int i = 0; i < n_lattices; ++i) {
        for (int k = 0; k < img; ++k) {
            LatticeRef& L = pa.lat[n];
            L.zeta = d_zetas[i];
            L.gamma = d_gammas[i];
            L.rows = rows[i];
            L.cols = cols[i];
            L.sign = k ? -1.0f : 1.0f;
            L.mirrored = k;
            pa.offset[n + 1] = pa.offset[n] + stream_len(rows[i], cols[i]);
            ++n;
        }
    }
    pa.n_lat = n;
    // Every element of the stream and every partial is written before it is read, so
    // nothing in the array has to start at zero.
    void* st = scratch;
    double* part = reinterpret_cast<double*>(scratch + stream_bytes);
    const int64_t fit = (int64_t)((kNoAllocScratchBytes - stream_bytes) / part_per_split);
    int n_split = choose_split(n_targets, n_elem, precision);
    if (n_split > fit) n_split = (int)fit;
    if (precision == FJ_PREC_FP64)
        FJ_TRY(pack_stream64(pa, (Elem64*)st, s));
    else
        FJ_TRY(pack_stream32(pa, (Elem32*)st, s));
    VindJob j;
    j.targets = d_targets;
    j.n_targets = n_targets;
    j.stream = st;
    j.n_elem = n_elem;
    j.n_split = n_split;
    j.part = part;
    j.n_links = n_links;
    FJ_TRY(vind_launch(j, precision, kernel, r_cut, s));
    return reduce_partials(part, n_split, n_targets, d_v_out, 0, 1.0, s);
}
