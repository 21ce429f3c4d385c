// fj_vind.cuh -- segment streams and the tiled all-pairs Biot-Savart sums.
//
// A lattice (rows+1) x (cols+1) of vertices carries two families of straight vortex
// filaments: chordwise zeta[k,l] -> zeta[k+1,l] and spanwise zeta[k,l] -> zeta[k,l+1]
// (aero/aic.py:277-282).  Both families are walked as polylines ("chains"): chordwise
// chain l visits zeta[0..rows, l], spanwise chain k visits zeta[k, 0..cols].  A stream
// is the concatenation of the chains of every source lattice; element i holds vertex i
// and the filament strength of the link i -> i+1 (aero/aic.py:284-287), and the last
// element of a chain is marked as a break.  Walking a chain, each (target, vertex)
// distance and its regularised inverse norm are computed once and shared by the two
// links that meet at the vertex -- the same numbers the reference computes twice, once
// per filament (aero/utils.py:614-619).
#pragma once

#include "fj_common.cuh"

namespace fj {

// FP64 stream element: 64 bytes.
struct __align__(16) Elem64 {
    double x, y, z;   // vertex
    double g;         // strength of link (this -> next); 0 on breaks
    double r0x, r0y, r0z;  // next - this, formed in FP64 as the reference does (y[1]-y[0])
    double q;         // epsilon kernel: EPSILON*|r0|^2*|r0|^2; cutoff/plain: |r0|^2; < 0: break
};

// FP32 stream element: 48 bytes.  Vertices are split hi+lo so that differences
// x - y are formed to FP32 relative precision even when |x|,|y| >> |x - y|.
struct __align__(16) Elem32 {
    float xh, yh, zh, g;   // g = strength / (4 pi)
    float xl, yl, zl, q;   // q as Elem64::q (FP32); < 0: break
    float r0x, r0y, r0z, pad;
};

// One source lattice for stream packing.
struct LatticeRef {
    const double* zeta;   // (rows+1, cols+1, 3)
    const double* gamma;  // (rows, cols); may be null when rows*cols == 0
    int rows, cols;
    float sign;           // +1, or -1 for a mirror image (aero/aic.py:306-308)
    int mirrored;         // 1: reflect vertices across the mirror plane
};

inline int64_t stream_len(int rows, int cols) {
    // chordwise chains (cols+1) of (rows+1) vertices + spanwise chains (rows+1) of (cols+1)
    return 2ll * (rows + 1) * (cols + 1);
}

struct MirrorPlane {
    double p[3];
    double nrm[3];
};

// Pack up to kMaxPack lattices into a stream (either precision).
constexpr int kMaxPack = 2 * 2 * FJ_MAX_SURF;  // (bound + wake) x (direct + image)

struct PackArgs {
    LatticeRef lat[kMaxPack];
    int64_t offset[kMaxPack + 1];
    int n_lat;
    int kernel;
    double r_cut;
    MirrorPlane mirror;
};

// Launch helpers (fj_vind.cu).
int pack_stream64(const PackArgs& a, Elem64* out, cudaStream_t s);
int pack_stream32(const PackArgs& a, Elem32* out, cudaStream_t s);

// Target-set x stream sum with per-split partials.  `part` has n_split * n_targets * 3
// doubles; `reduce_partials` then sums them in split order into `out` (+= when
// accumulate != 0).
struct VindJob {
    const double* targets;  // (n_targets, 3)
    int64_t n_targets;
    const void* stream;     // Elem64* or Elem32*
    int64_t n_elem;
    int n_split;
    double* part;           // (n_split, n_targets, 3)
    int64_t n_links;        // filaments in the stream (for pair counting)
    double* out;            // (n_targets, 3) result of the reduction (batched launches)
    int accumulate;         // batched reduction: 1 adds the sum to out, 0 overwrites out
};

// A stream-packing job of a batched launch: lattices -> elements at `out`.
struct PackJob {
    PackArgs a;
    void* out;
};

// Batched launches (one kernel for many jobs; tables in device memory).
//  vind: CTAs of job j are cta0[j] .. cta0[j+1]-1 (ctas_x(j) * n_split(j) of them);
//  all jobs of one launch share precision and kernel.
int vind_launch_jobs(const VindJob* d_jobs, const int64_t* d_cta0, int n_jobs, int64_t total_ctas, double pairs,
                     int precision, int kernel, double r_cut, cudaStream_t s, bool persistent = false,
                     int tile = 0);
int pack_jobs(const PackJob* d_jobs, int n_jobs, int64_t max_elem, int precision, cudaStream_t s);
int reduce_jobs(const VindJob* d_jobs, int n_jobs, int64_t max_targets, cudaStream_t s);
// CTAs of one sum (target tiles x splits), for building cta0; tile = targets per thread of
// the FP32 sum (2 or 4; 0 = 2), ignored for FP64.
int64_t vind_ctas(int64_t n_targets, int n_split, int precision, int tile = 0);

// filaments of an (rows, cols) lattice: rows(cols+1) chordwise + (rows+1)cols spanwise
inline int64_t lattice_links(int rows, int cols) {
    return (int64_t)rows * (cols + 1) + (int64_t)(rows + 1) * cols;
}

// tile: FP32 targets per thread (2 or 4); 0 takes the tuned table's choice for the shape.
int vind_launch(const VindJob& job, int precision, int kernel, double r_cut, cudaStream_t s, int tile = 0);
int reduce_partials(const double* part, int n_split, int64_t n_targets, double* out,
                    int accumulate, double scale, cudaStream_t s);
int choose_split(int64_t n_targets, int64_t n_elem, int precision);
// FP32 targets per thread for a shape: 4 where the autotuner found the wide tile faster,
// else 2 (FP64: 2).
int choose_tile(int64_t n_targets, int64_t n_elem, int precision);
// A tuned table entry: the split count, with bit 12 set when the wide tile won.
int encode_tuned(int split, int tile);
// The wave-filling rule choose_split falls back to where no tuned entry exists.
int heuristic_split(int64_t n_targets, int64_t n_elem, int precision);

// Tuned split counts (and, FP32, the tile: bit 12 set for four targets per thread), by
// precision (0 FP64, 1 FP32), log2 of the target count and log2 of the stream length;
// 0 = not tuned.  A published table is immutable.
constexpr int kTuneTargetBuckets = 24, kTuneElemBuckets = 28;
struct TuneTable {
    int16_t split[2][kTuneTargetBuckets][kTuneElemBuckets];
};
const TuneTable* tune_table();
void tune_publish(const TuneTable* t);
int tune_bucket_targets(int64_t n_targets);
int tune_bucket_elem(int64_t n_elem);
int split_bound(int64_t n_targets, int64_t n_elem_max, int precision);

}  // namespace fj
