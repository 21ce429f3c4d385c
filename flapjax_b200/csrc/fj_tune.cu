// fj_tune.cu -- autotuner of the Biot-Savart sum launches.
//
// A sum of n_targets points over a stream of n_elem filament elements is launched as
// (target tiles) x (splits) CTAs, each split summing a slice of the stream into its own
// partials, reduced afterwards.  The split count trades parallelism against partial
// traffic and the last wave's fill.  choose_split takes it from a rule that fills whole
// waves; fj_autotune_vind measures instead: for each requested shape it builds a
// synthetic lattice of that stream length (a flat grid with seeded jitter, so the stream
// has the real element layout, chain breaks included) and seeded targets above it, times
// the sum + reduction at candidate split counts with CUDA events, and publishes the
// fastest into a new immutable table (keyed by precision, log2 targets, log2 stream
// length) that choose_split consults from then on.  The FP32 sums are also timed with four
// targets per thread instead of two (the tile shape: twice the targets share each staged
// filament element, at twice the registers and half the resident CTAs); the table records
// which tile won beside the split.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fj_vind.cuh"

namespace fj {
namespace {

__device__ __forceinline__ double hash01(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

// zeta (rows+1, cols+1, 3): a 1 x 8 grid with 1 % jitter; gamma in [0.5, 1.5).
__global__ void tune_lattice_kernel(double* zeta, double* gamma, int rows, int cols) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nv = (int64_t)(rows + 1) * (cols + 1);
    if (i < nv) {
        const int r = (int)(i / (cols + 1)), c = (int)(i % (cols + 1));
        zeta[i * 3 + 0] = (double)r / rows + 0.01 * (hash01(3 * i) - 0.5) / rows;
        zeta[i * 3 + 1] = 8.0 * c / cols + 0.01 * (hash01(3 * i + 1) - 0.5) / cols;
        zeta[i * 3 + 2] = 0.02 * hash01(3 * i + 2);
    }
    if (i < (int64_t)rows * cols) gamma[i] = 0.5 + hash01(i + 0x9e3779b97f4a7c15ull);
}

// Targets spread over the lattice's box, 0.01 .. 0.5 above it.
__global__ void tune_targets_kernel(double* t, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    t[i * 3 + 0] = hash01(7 * i + 1);
    t[i * 3 + 1] = 8.0 * hash01(7 * i + 2);
    t[i * 3 + 2] = 0.01 + 0.49 * hash01(7 * i + 3);
}

void lattice_dims(int64_t n_elem, int* rows, int* cols) {
    // stream length 2 (rows+1)(cols+1); spans up to 128 panels, as the wings here
    const int64_t half = std::max<int64_t>(4, n_elem / 2);
    int c = (int)std::min<int64_t>(128, std::max<int64_t>(1, (int64_t)std::sqrt((double)half) - 1));
    int r = (int)std::max<int64_t>(1, half / (c + 1) - 1);
    *rows = r;
    *cols = c;
}

struct ShapeWs {
    size_t targets, zeta, gamma, stream, part, out, total;
};

ShapeWs shape_ws(int precision, int64_t n_targets, int64_t n_elem) {
    int rows, cols;
    lattice_dims(n_elem, &rows, &cols);
    const int64_t ne = stream_len(rows, cols);
    Arena a(nullptr, 0);
    ShapeWs w{};
    w.targets = (size_t)n_targets * 3;
    w.zeta = (size_t)(rows + 1) * (cols + 1) * 3;
    w.gamma = (size_t)rows * cols;
    w.stream = (size_t)ne;
    w.part = (size_t)split_bound(n_targets, ne, precision) * n_targets * 3;
    w.out = (size_t)n_targets * 3;
    a.carve<double>(w.targets);
    a.carve<double>(w.zeta);
    a.carve<double>(w.gamma);
    if (precision == FJ_PREC_FP64) a.carve<Elem64>(w.stream);
    else a.carve<Elem32>(w.stream);
    a.carve<double>(w.part);
    a.carve<double>(w.out);
    w.total = a.used + 256;
    return w;
}

}  // namespace
}  // namespace fj

using namespace fj;

extern "C" {

int fj_autotune_vind_workspace_size(int precision, const int64_t* n_targets, const int64_t* n_elem, int n_shapes,
                                    size_t* bytes) {
    if (!bytes || n_shapes < 0 || (n_shapes > 0 && (!n_targets || !n_elem)))
        return fail(FJ_ERR_SHAPE, "autotune: bad arguments");
    size_t need = 256;
    for (int i = 0; i < n_shapes; ++i) {
        if (n_targets[i] <= 0 || n_elem[i] <= 0) return fail(FJ_ERR_SHAPE, "autotune: shape %d is empty", i);
        need = std::max(need, shape_ws(precision, n_targets[i], n_elem[i]).total);
    }
    *bytes = need;
    return FJ_OK;
}

int fj_autotune_vind(int precision, int kernel, double r_cut, const int64_t* n_targets, const int64_t* n_elem,
                     int n_shapes, int* chosen, int* heuristic, double* chosen_ms, double* heuristic_ms, void* d_ws,
                     size_t ws_bytes, fj_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (precision != FJ_PREC_FP64 && precision != FJ_PREC_MIXED)
        return fail(FJ_ERR_SHAPE, "autotune: precision %d", precision);
    size_t need = 0;
    FJ_TRY(fj_autotune_vind_workspace_size(precision, n_targets, n_elem, n_shapes, &need));
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "autotune workspace %zu < %zu", ws_bytes, need);
    TuneTable* table = new TuneTable();
    if (const TuneTable* old = tune_table()) *table = *old;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = cuda_status(cudaEventCreate(&e0), "autotune event");
    if (st == FJ_OK) st = cuda_status(cudaEventCreate(&e1), "autotune event");
    for (int i = 0; i < n_shapes && st == FJ_OK; ++i) {
        int rows, cols;
        lattice_dims(n_elem[i], &rows, &cols);
        const int64_t ne = stream_len(rows, cols), nt = n_targets[i];
        Arena a(d_ws, ws_bytes);
        double* targets = a.carve<double>((size_t)nt * 3);
        double* zeta = a.carve<double>((size_t)(rows + 1) * (cols + 1) * 3);
        double* gamma = a.carve<double>((size_t)rows * cols);
        void* strm = precision == FJ_PREC_FP64 ? (void*)a.carve<Elem64>(ne) : (void*)a.carve<Elem32>(ne);
        const int bound = split_bound(nt, ne, precision);
        double* part = a.carve<double>((size_t)bound * nt * 3);
        double* out = a.carve<double>((size_t)nt * 3);
        const int64_t nv = (int64_t)(rows + 1) * (cols + 1);
        tune_lattice_kernel<<<(unsigned)((nv + 255) / 256), 256, 0, s>>>(zeta, gamma, rows, cols);
        tune_targets_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(targets, nt);
        note_launch(2);
        st = cuda_status(cudaGetLastError(), "autotune fill kernels");
        if (st != FJ_OK) break;
        PackArgs pa{};
        pa.lat[0] = LatticeRef{zeta, gamma, rows, cols, 1.0f, 0};
        pa.offset[0] = 0;
        pa.offset[1] = ne;
        pa.n_lat = 1;
        pa.kernel = kernel;
        pa.r_cut = r_cut;
        st = precision == FJ_PREC_FP64 ? pack_stream64(pa, (Elem64*)strm, s) : pack_stream32(pa, (Elem32*)strm, s);
        if (st != FJ_OK) break;
        const int h = heuristic_split(nt, ne, precision);
        std::vector<int> cand = {1, h, h / 4, h / 2, (3 * h) / 2, 2 * h, 3 * h, 4 * h};
        for (int& c : cand) c = std::max(1, std::min(c, bound));
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        int best = h, best_tile = 2;
        float best_ms = 0.0f, h_ms = 0.0f;
        // FP32: each split count with two and with four targets per thread
        std::vector<std::pair<int, int>> trials;
        for (int sp : cand) {
            trials.push_back({sp, 2});
            if (precision == FJ_PREC_MIXED) trials.push_back({sp, 4});
        }
        for (const auto& trial : trials) {
            const int sp = trial.first, tile = trial.second;
            VindJob job{targets, nt, strm, ne, sp, part, ne, out};
            float t = 1e30f;
            for (int rep = 0; rep < 4 && st == FJ_OK; ++rep) {
                float ms = 0.0f;
                st = cuda_status(cudaEventRecord(e0, s), "autotune event");
                if (st == FJ_OK) st = vind_launch(job, precision, kernel, r_cut, s, tile);
                if (st == FJ_OK) st = reduce_partials(part, sp, nt, out, 0, 1.0, s);
                if (st == FJ_OK) st = cuda_status(cudaEventRecord(e1, s), "autotune event");
                if (st == FJ_OK) st = cuda_status(cudaEventSynchronize(e1), "autotune sync");
                if (st == FJ_OK) st = cuda_status(cudaEventElapsedTime(&ms, e0, e1), "autotune timing");
                if (rep > 0) t = std::min(t, ms);  // the first run warms up
            }
            if (st != FJ_OK) break;
            if (sp == h && tile == 2) h_ms = t;
            // a challenger must be 2 % faster; the rule's split with the default tile wins ties
            if (best_ms == 0.0f || t < best_ms * 0.98f || (t <= best_ms * 1.02f && sp == h && tile == 2)) {
                best = sp;
                best_tile = tile;
                best_ms = t;
            }
        }
        if (st != FJ_OK) break;
        table->split[precision == FJ_PREC_FP64 ? 0 : 1][tune_bucket_targets(nt)][tune_bucket_elem(ne)] =
            (int16_t)encode_tuned(best, best_tile);
        if (chosen) chosen[i] = encode_tuned(best, best_tile);
        if (heuristic) heuristic[i] = h;
        if (chosen_ms) chosen_ms[i] = best_ms;
        if (heuristic_ms) heuristic_ms[i] = h_ms;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st != FJ_OK) {
        delete table;
        return st;
    }
    tune_publish(table);  // earlier tables stay allocated: readers hold no lock
    return FJ_OK;
}

int fj_autotune_table_size(int* n_entries) {
    if (!n_entries) return fail(FJ_ERR_SHAPE, "autotune: null argument");
    *n_entries = (int)(sizeof(TuneTable) / sizeof(int16_t));
    return FJ_OK;
}

int fj_autotune_get(int16_t* entries, int n_entries) {
    if (!entries || n_entries != (int)(sizeof(TuneTable) / sizeof(int16_t)))
        return fail(FJ_ERR_SHAPE, "autotune: table has %d entries", (int)(sizeof(TuneTable) / sizeof(int16_t)));
    const TuneTable* t = tune_table();
    if (t) std::copy(&t->split[0][0][0], &t->split[0][0][0] + n_entries, entries);
    else std::fill(entries, entries + n_entries, (int16_t)0);
    return FJ_OK;
}

int fj_autotune_set(const int16_t* entries, int n_entries) {
    if (n_entries == 0 && entries == nullptr) {
        tune_publish(nullptr);
        return FJ_OK;
    }
    if (!entries || n_entries != (int)(sizeof(TuneTable) / sizeof(int16_t)))
        return fail(FJ_ERR_SHAPE, "autotune: table has %d entries", (int)(sizeof(TuneTable) / sizeof(int16_t)));
    // entries: 0 (not tuned) or a split count in 1..1024, the FP32 block's with bit 12 for
    // the four-target tile
    const int half = n_entries / 2;
    for (int i = 0; i < n_entries; ++i) {
        const int v = entries[i], split = v & 0xFFF, extra = v & ~0xFFF;
        const bool ok = v >= 0 && split <= 1024 && (extra == 0 || (extra == 0x1000 && i >= half && split >= 1));
        if (!ok) return fail(FJ_ERR_SHAPE, "autotune: entry %d = %d", i, v);
    }
    TuneTable* t = new TuneTable();
    std::copy(entries, entries + n_entries, &t->split[0][0][0]);
    tune_publish(t);
    return FJ_OK;
}

}  // extern "C"
