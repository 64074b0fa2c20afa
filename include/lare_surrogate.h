/*
 * lare_surrogate.h - device kernels of the learned conduction surrogate.
 *
 * The surrogate has no counterpart in the reference (Lare3d integrates
 * conduction only with RKL2, conduct.f90:299-416); it is the learned form
 * that sits beside the plain RKL2 step, which stays both its fallback and the
 * arbiter of its accuracy.  A 4-layer 3-D convolutional network (3^3 kernels, 32 channels,
 * bf16 weights and activations, FP32 accumulation on the tensor cores) maps
 * a window of (T, rho, b-hat) to the temperature change of one RKL2 step on
 * the window's centre (valid convolutions: each layer trims one cell per
 * face, so a window of edge w predicts the central (w - 8)^3).
 *
 * All pointers are device pointers; every call enqueues work on `stream`
 * (a cudaStream_t, NULL = default stream) and returns 0 or a negative
 * LARE_E* code from lare_gpu.h.  Tensors are channels-last:
 *   activations  [batch][d][d][d][channels]   bf16
 *   weights      [27][cout][cin]   bf16, tap t = (dz*3 + dy)*3 + dx
 * Engine arrays are addressed as lare_gpu_field_device returns them: element
 * (i, j, k) (Fortran indices) at origin[i + sx*j + sxy*k], FP64 or FP32 by
 * elem_bytes.  Grid cell (x, y, z), 0-based, is Fortran (x+1, y+1, z+1).
 */
#ifndef LARE_SURROGATE_H
#define LARE_SURROGATE_H

#ifdef __cplusplus
extern "C" {
#endif

/*
 * y[b][o][co] = act( sum_{t,ci} w[t][co][ci] * x[b][o + d(t) - pad][ci] + bias[co] )
 * x: [nb][din]^3[cin] bf16 (zero outside), y: [nb][dout]^3[cout] bf16 or FP32
 * (out_f32), dout = din - 2 + 2*pad with pad 0 (valid) or 2 (full).
 * act = ReLU if relu; if mask is given (same layout as a bf16 y) the result is
 * multiplied by (mask > 0) (the ReLU derivative, for the backward pass).
 * bias may be NULL.  Backward-data is this call with pad = 2 on the output
 * gradient and the tap-flipped, transposed weights of lare_sur_pack.
 * (cin, cout) in {(16,32), (32,32), (32,8), (32,1)}; (32,1) is the
 * network's output layer (FP32 output, no mask), computed with the nine
 * in-plane taps in the MMA's N dimension.
 */
int lare_sur_conv(int cin, int cout, int relu, int out_f32, const void* x, int din, int pad, const void* w,
                  const float* bias, void* y, int dout, int nb, const void* mask, void* stream);

/*
 * Selects the convolution engine: 1 (default) = tcgen05.mma on the 5th-
 * generation tensor cores with accumulators in tensor memory; 0 = the
 * warp-level mma.sync kernel.  Both compute the same sums (FP32
 * accumulation, summation order differs).  Process-wide.
 */
int lare_sur_set_engine(int tensor_cores);

/*
 * Sticky status of the tensor-core kernels: 0, or a bit mask of device-side
 * failures (1 = a wait on the tensor cores ran out; the kernel skipped its
 * remaining work).  Synchronises the device; clear != 0 resets the word.
 */
int lare_sur_status(int clear);

/*
 * Weight and bias gradients of a valid conv (din = dout + 2):
 * dw[t][co][ci] = sum_{b,o} dy[b][o][co] * x[b][o + d(t)][ci],
 * db[co] = sum_{b,o} dy[b][o][co] (db may be NULL), FP32, deterministic
 * (fixed-order sums).  work: FP32 scratch of lare_sur_conv_wgrad_work()
 * floats.  (cin, cout) in {(16,32), (32,32), (32,16)}.
 */
int lare_sur_conv_wgrad(int cin, int cout, const void* dy, const void* x, int din, int dout, int nb, float* work,
                        float* dw, float* db, void* stream);
long long lare_sur_conv_wgrad_work(int cin, int cout, int dout, int nb);

/*
 * Mean squared error of channel 0 of pred ([count][pc] FP32) against target
 * ([count] FP32): loss[0] = mean((pred - target)^2); dy ([count][cpad] bf16)
 * receives 2 (pred - target) / count in channel 0 and zeros elsewhere.
 * work: FP32 scratch of (count + 255) / 256 floats.
 */
int lare_sur_mse(const float* pred, int pc, const float* target, long long count, int cpad, float* loss, void* dy,
                 float* work, void* stream);

/* Adam step on n FP32 parameters (bias-corrected, step t >= 1). */
int lare_sur_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                  int t, void* stream);

/*
 * Pack FP32 master weights wm [27][cout][cin] into the bf16 forward layout
 * wf [27][cout_f][cin] (the first cout_f <= cout output channels) and, if wb
 * is not NULL, the backward-data layout wb [27][cin][cout] (taps flipped,
 * t' = 26 - t, and transposed).
 */
int lare_sur_pack(const float* wm, int cin, int cout, int cout_f, void* wf, void* wb, void* stream);

/*
 * Features of the resident state: feat [5][nz][ny][nx] FP32 =
 * (T * t_scale, rho * rho_scale, b-hat x, y, z) with T from energy as in
 * conduct.f90:68 and b-hat the unit vector of the face fields averaged to the
 * cell centre.  If tout is not NULL it receives T ([nz][ny][nx] FP32) when
 * tmode = 0 and T - tout (in place) when tmode = 1.  feat may be NULL.
 */
int lare_sur_extract(int elem_bytes, const void* energy, const void* rho, const void* bx, const void* by,
                     const void* bz, int sx, int sxy, int nx, int ny, int nz, double gamma, double xi_n,
                     double ionise_pot, float t_scale, float rho_scale, float* feat, float* tout, int tmode,
                     void* stream);

/*
 * Gather nb windows of edge win from feature stores [S][5][nz][ny][nx] at
 * org[4*b] = (store s, x0, y0, z0) (x and y wrap periodically, z is
 * clamped) into x [nb][win]^3[16] bf16: channels 0..4 are the five features
 * rounded to bf16, channels 5 and 6 are 256 x the rounding remainders of
 * features 0 and 1 (T and rho), channels 7..15 are zero.  If tgt is not
 * NULL, also the central (win - 2*halo)^3 of the target stores
 * tstore [S][nz][ny][nx], times tscale, into tgt [nb][(win - 2*halo)^3].
 */
int lare_sur_gather(const float* store, int nx, int ny, int nz, const int* org, int nb, int win, int halo, void* x,
                    const float* tstore, float tscale, float* tgt, void* stream);

/*
 * energy(cell) += out_scale * pred[b][l][0] for every window b and every
 * cell l of its central (pw)^3 (pred [nb][pw^3][pc] FP32), the cell being
 * org[4*b+1..3] + halo + l (x, y wrapped).  Windows' centres must not overlap.
 */
int lare_sur_apply(int elem_bytes, void* energy, int sx, int sxy, int nx, int ny, int nz, const float* pred, int pc,
                   const int* org, int nb, int pw, int halo, double out_scale, void* stream);

/*
 * Copy up to 8 arrays of a full-height column of the grid into a window
 * engine: dst(i, j, k) = src(wrap_x(x0 + i), wrap_y(y0 + j), k) for the whole
 * padded box of the window (Fortran i in -2..wnx+2, j in -2..wny+2, k in
 * -2..nz+2), with wrap_x(i) = ((i - 1) mod nx) + 1.  The window keeps the
 * source's nz.  src and dst hold n pointers each.
 */
int lare_sur_copy_column(int elem_bytes, const void* const* src, int sx, int sxy, int nx, int ny, void* const* dst,
                         int wsx, int wsxy, int wnx, int wny, int nz, int x0, int y0, int n, void* stream);

/*
 * Re-check of patches against a plain-RKL2 window: for each patch p of edge
 * `patch` at grid cells (px0 + a*patch, py0 + b*patch, pz0 + c*patch)
 * (x, y wrapped), a < npx, b < npy, c < npz, p = a + npx*(b + npy*c),
 * err[p] = max |T - T_w| / |T_w| over the patch (T from the main energy,
 * T_w from the window energy at the same cell, the window of wnx x wny
 * columns having its cell (1, 1, 1) at grid cell (x0, y0, 0), x0 <= px0,
 * y0 <= py0).  Where err[p] > bound the patch is rejected: its energy is
 * replaced by the window's and *n_rejected is incremented.
 */
int lare_sur_recheck(int elem_bytes, void* energy, int sx, int sxy, int nx, int ny, const void* energy_w, int wsx,
                     int wsxy, int wnx, int wny, int x0, int y0, int px0, int py0, int pz0, int npx, int npy, int npz,
                     int patch, double gamma, double xi_n, double ionise_pot, double bound, float* err,
                     int* n_rejected, void* stream);

#ifdef __cplusplus
}
#endif

#endif
