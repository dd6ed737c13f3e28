// Vector kernels of the Krylov drivers (replace the deal.II
// LinearAlgebra::distributed::Vector<.., MemorySpace::CUDA> BLAS-1 calls of
// include/solver.cuh:1830-1999 and copy_vector, :64-78).  Reductions are
// two-stage with a fixed grid, so every dot product is deterministic.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "intdiv.cuh"

namespace tps {

constexpr int kRedBlocks = 592;   // 4 x 148 SMs
constexpr int kRedThreads = 512;

// Index map from a lexicographic vector to a level vector whose rows of N1
// entries are sy apart (sy == N1: identity).
struct PadMap {
  int N1;
  int64_t sy;
  uint32_t m, s;  // i / N1 == (i * m) >> s (magic_div), for i < 2^31
};

inline PadMap make_padmap(int N1, int64_t sy)
{
  PadMap pm{N1, sy, 0, 0};
  magic_div(static_cast<uint32_t>(N1), pm.m, pm.s);
  return pm;
}

// Device-resident scalars of the CG iteration (no host round trip inside an
// iteration, so one iteration can be captured in a CUDA graph).
struct CGScalars {
  double rz;      // r . z
  double pq;      // p . A p
  double alpha;
  double beta;
  double rr;      // r . r
  double zq;      // z . q
  double rz_new;
  double bb;      // b . b
  int breakdown;  // set when p.Ap <= 0 or a non-finite value appears
  int pad;
};

// dst[i] = (Tout) src[i]; round32 != 0 rounds through FP32 first
// n 32-bit words src -> dst by one small kernel; dst may be host-mapped
// memory, so a small result reaches the host without a copy-engine transfer
// (which would queue behind large copies on other streams)
cudaError_t launch_copy_words(const void *src, void *dst, int n_words, cudaStream_t s);
// one CTA whose bounded mbarrier wait runs out after `cycles` SM cycles and
// sets *err (the timeout path of the smoother kernels, exercised without a fault)
cudaError_t launch_wait_timeout_selftest(int *err, long long cycles, cudaStream_t s);
cudaError_t launch_convert_f64_to_f32(float *dst, const double *src, int64_t n, cudaStream_t s);
cudaError_t launch_convert_f32_to_f64(double *dst, const float *src, int64_t n, cudaStream_t s);
cudaError_t launch_copy_f64(double *dst, const double *src, int64_t n, int round32, cudaStream_t s);
// boundary rows of a lexicographic level vector: dst_b = src_b
cudaError_t launch_copy_boundary(void *dst, const void *src, int dim, int N1, int elem_bytes,
                                 cudaStream_t s);
// partial dot products into partial[kRedBlocks * n_dots]
cudaError_t launch_dot_f64(const double *a, const double *b, int64_t n, double *partial,
                           cudaStream_t s);
// reduce partial sums; out[i] = sum of partial[i*kRedBlocks ...]
cudaError_t launch_reduce(const double *partial, int n_dots, double *out, cudaStream_t s);

// --- fused CG steps (flexible CG, FP64 outer) ---------------------------
// r = b - A x was formed by the operator; rr, and the V-cycle input d
// (FP32, FP64, or FP64 rounded through FP32) are produced from r.
cudaError_t launch_cg_init(const double *r, const double *b, void *d, int d_kind, PadMap pm,
                           int64_t n, double *partial, cudaStream_t s);
// finalize: sc.rr = sum, sc.bb = sum
cudaError_t launch_cg_finalize_init(const double *partial, CGScalars *sc, cudaStream_t s);
// p = z, partial(r.z) ; z in V-cycle precision
cudaError_t launch_cg_first_direction(double *p, const void *z, int z_kind, PadMap pm,
                                      const double *r, int64_t n, double *partial, cudaStream_t s);
cudaError_t launch_cg_finalize_rz(const double *partial, CGScalars *sc, cudaStream_t s);
// partial(p.q) then alpha = rz / pq
// alpha from `count` partial sums of p.q formed elsewhere (the fused
// operator kernel), summed in a fixed order
cudaError_t launch_cg_alpha_partials(const double *partial, int count, CGScalars *sc, cudaStream_t s);
cudaError_t launch_cg_alpha(const double *p, const double *q, int64_t n, double *partial,
                            CGScalars *sc, cudaStream_t s);
// x += alpha p, r -= alpha q, d = conv(r), partial(r.r)
cudaError_t launch_cg_update_xr(double *x, double *r, const double *p, const double *q, void *d,
                                int d_kind, PadMap pm, int64_t n, double *partial,
                                const CGScalars *sc, cudaStream_t s);
cudaError_t launch_cg_finalize_rr(const double *partial, CGScalars *sc, cudaStream_t s);
// partial(z.q), partial(z.r) then beta = -alpha zq / rz, rz = z.r
cudaError_t launch_cg_beta(const void *z, int z_kind, PadMap pm, const double *q, const double *r,
                           int64_t n, double *partial, CGScalars *sc, cudaStream_t s);
// p = z + beta p
cudaError_t launch_cg_update_p(double *p, const void *z, int z_kind, PadMap pm, int64_t n,
                               const CGScalars *sc, cudaStream_t s);

// generic FP64 helpers for the GMRES driver
cudaError_t launch_axpy_f64(double *y, double a, const double *x, int64_t n, cudaStream_t s);
cudaError_t launch_scale_f64(double *y, double a, int64_t n, cudaStream_t s);
cudaError_t launch_sub_f64(double *dst, const double *a, const double *b, int64_t n,
                           cudaStream_t s);  // dst = a - b
// V-cycle input from an FP64 vector and FP64 output from the V-cycle result
cudaError_t launch_to_vcycle(void *d, int d_kind, PadMap pm, const double *src, int64_t n,
                             cudaStream_t s);
cudaError_t launch_from_vcycle(double *dst, const void *z, int z_kind, PadMap pm, int64_t n,
                               cudaStream_t s);
cudaError_t launch_fill(void *dst, int elem_bytes, int64_t n, cudaStream_t s);  // zero

// --- batched solves: device-side control of one graph launch -------------
// State of the batched CG loop (device memory, one entry per system).
struct BatchLoop {
  CGScalars *const *sc;  // per-system CG scalars
  int *iters;            // iterations done
  int *active;           // still iterating
  double *bnorm;         // ||b|| (1 if b = 0)
  double *hist;          // relative residual history, hist_len per system
  int n, hist_len, max_iter;
  double rel_tol;
};
// first = 1: after the initial residual (iteration 0); first = 0: after one
// more iteration of every active system.  Updates the state and sets the
// while-condition `loop` to "some system still active".
cudaError_t launch_batch_check(BatchLoop b, int first, cudaGraphConditionalHandle loop, cudaStream_t s);
// sets the if-condition of every system from its active flag (start of a loop
// body); the handles are passed by value (kernel parameters), up to 256
constexpr int kBatchMax = 256;
struct BatchConds {
  cudaGraphConditionalHandle h[kBatchMax];
};
cudaError_t launch_batch_select(const int *active, const BatchConds &cond, int n, cudaStream_t s);

}  // namespace tps
