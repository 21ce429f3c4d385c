// fj_common.cuh -- shared definitions of libfj_uvlm (status handling, constants, PODs).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "fj_uvlm.h"

namespace fj {

// utils/constants.py:16 (EPSILON), :19 (R_CUTOFF)
constexpr double kEps = 1e-7;
constexpr double kRCutoffDefault = 1e-4;
constexpr double kPi = 3.14159265358979323846;
constexpr double kFourPi = 4.0 * kPi;

// Sine of the angle below which the FP32 kernel treats a (target, segment) pair as
// collinear and returns exactly zero, as the FP64 epsilon kernel does to within its
// rounding noise.  FP32 resolves the cross product r1 x r2 to about 1e-7 |r1||r2|;
// this threshold sits a decade above that floor.
constexpr float kCollinearSin = 4e-6f;

void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

// Count of kernels this library has launched (read through fj_launch_count).
void note_launch(int n = 1);
int64_t launch_count();

// True while fj_profile_begin/_end bracket a region (its event records cannot be
// captured into a CUDA graph).
bool prof_active();

// Raise a kernel's dynamic shared-memory limit on the current device to at least
// `bytes`.  The limit only ever grows, under a lock, so host threads launching the same
// kernel on different streams never lower each other's limit between set and launch.
int allow_dynamic_smem(const void* func, size_t bytes);

// Opt-in timing of the Biot-Savart sum kernels with CUDA events on their stream
// (fj_profile_begin / fj_profile_end).  prof_start returns -1 when profiling is off.
int prof_start(cudaStream_t s);
void prof_stop(int slot, cudaStream_t s, double pairs, bool fp64);

inline int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return FJ_OK;
    return fail(FJ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define FJ_TRY(expr)                        \
    do {                                    \
        int _st = (expr);                   \
        if (_st != FJ_OK) return _st;       \
    } while (0)

#define FJ_CUDA(expr) FJ_TRY(::fj::cuda_status((expr), #expr))
#define FJ_LAUNCH_CHECK(what) FJ_TRY(::fj::cuda_status(cudaGetLastError(), what))

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Bump allocator over a caller-provided workspace.  Carving is pure arithmetic, so the
// same sequence of carve() calls yields the same layout on every call.
struct Arena {
    char* base;
    size_t cap;
    size_t used;
    explicit Arena(void* b = nullptr, size_t c = 0) : base((char*)b), cap(c), used(0) {}
    template <typename T>
    T* carve(size_t count) {
        used = align_up(used, 256);
        T* p = base ? (T*)(base + used) : nullptr;
        used += count * sizeof(T);
        return p;
    }
    bool fits() const { return used <= cap; }
};

// Pair counting convention for roofline reports: one (target, segment) kernel
// evaluation.  Exposed for the benchmark through fj_stats.
struct Dims {
    int m, n, m_star;
};

}  // namespace fj
