/*
 * oi_b200.h -- C ABI of the B200 aerial-image engine (liboi_b200.so).
 *
 * The reference exposes its imaging path as Python functions over torch tensors; it has no native ABI.
 * Each entry point below replaces the numerical core of one of those functions, so a binding (ctypes,
 * cffi, pybind) can call it with plain device pointers:
 *
 *   oi_band_spectrum      <- Scatter.CalculateSpectrum                    (Scatter.py:10-35)
 *   oi_abbe_pupils        <- the per-source-point pupil of CalculateAbbeImage (CalculateAerialImage.py:46-75)
 *   oi_coherent_coarse    <- the |fft2(.)|^2 accumulation of CalculateAbbeImage (CalculateAerialImage.py:76-92)
 *                            and of CalculateAerialImage_SOCS               (CalculateAerialImage_SOCS.py:5-10)
 *   oi_coarse_to_image    <- the final fftshift + normalisation of both     (CalculateAerialImage.py:89-92,
 *                                                                             CalculateAerialImage_SOCS.py:10)
 *   oi_tcc_pupils64       <- the shifted-pupil matrix of CalculateTCCMatrix  (CalculateTCCMatrix.py:17-51)
 *   oi_abbe_pupils_pol / oi_tcc_pupils64_pol
 *                         <- the same with a Jones vector per source point: Calc_PolarizationMap's typed maps
 *                            (Source.py:183-221) and the states of a CoherencyMatrix (README.md:45)
 *   oi_tcc_assemble64     <- GetTCCMatrix                                    (CalculateTCCMatrix.py:58-75)
 *   oi_eig_topk64         <- the SVD and truncation of DecomposeTCC_SOCS     (DecomposeTCC_SOCS.py:7-9)
 *   oi_band_spectrum_fft / oi_coherent_coarse_fft / oi_coarse_to_image_fft
 *                         <- the same three stages in FFT form (power-of-two grids)
 *   oi_spectrum_to_image(_fft) <- the synthesis half of the two above
 *   oi_coherent_coarse_tc <- the |fft2(.)|^2 accumulation again, split-BF16x3 on tensor cores (tcgen05)
 *   oi_band_spectrum_tc(_sym) / oi_coarse_to_image_tc / oi_rows_fwd_tc(_half) / oi_rows_inv_tc
 *                         <- the N-point stages with their row passes on the tensor cores (split-BF16x3 form)
 *   oi_synth_tc_constants / oi_synth_tiles_tc / oi_coarse_to_image_tcs
 *                         <- the final transform of CalculateAerialImage_SOCS.py:7-10 on the intensity's band,
 *                            coarse spectrum and column synthesis as tensor-core GEMMs
 *   oi_coherent_adjoint   <- (no counterpart: the reference differentiates through torch autograd)
 *   oi_twiddle            <- (no counterpart: fills the phase tables the transforms read)
 *
 * Conventions
 *   - Every function returns 0 on success or a negative OI_E* status; oi_last_error() describes the last
 *     failure on the calling thread.  Nothing aborts the process.
 *   - All pointers are device pointers owned by the caller; nothing here allocates device memory.
 *   - `stream` is a cudaStream_t passed as void*; all work is enqueued on it and nothing synchronises, except
 *     where an entry point says so (oi_eig_topk64, oi_device_status).
 *   - float2 / double2 are interleaved (re, im) pairs, the layout of torch complex64 / complex128.
 *   - Frequencies are centred integers: band row i means frequency m0r + i (cycles per period).
 *   - Image convention: out[y][x] = sum_fields w * |sum_m P(m) c(m) exp(-2 pi i (m_r y/Ny + m_c x/Nx))|^2
 *     with c(m) = 1/(Ny Nx) sum_{y,x} h[y][x] exp(+2 pi i (m_r y/Ny + m_c x/Nx)).  This equals the
 *     reference's fftshift(sum |fft2(...)|^2) * dfdg^2 output index for index, for even and odd sizes.
 */
#ifndef OI_B200_H
#define OI_B200_H

#if defined(__GNUC__)
#define OI_API __attribute__((visibility("default")))
#else
#define OI_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  OI_OK = 0,
  OI_EINVAL = -1,      /* invalid argument (sizes, null pointers, unsupported kind) */
  OI_ECUDA = -2,       /* a CUDA launch or runtime call failed */
  OI_ERANGE = -3,      /* a size is above a compiled limit */
};

/* Field kinds for oi_band_spectrum. */
enum {
  OI_FIELD_REAL_F32 = 0,     /* float  [batch][ny][nx]            (thin real transmission)          */
  OI_FIELD_COMPLEX_C64 = 1,  /* float2 [batch][ny][nx][nch]       (the reference's ScatterField)    */
  OI_FIELD_U8 = 2,           /* uint8  [batch][ny][nx], raw value (fold any grey scaling into `scale`) */
};

OI_API const char* oi_last_error(void);
OI_API int oi_version(void);

/*
 * Phase table  out[a][b] = scale * exp(sign * 2 pi i * ((a + a0) * (b + b0) mod n) / n)
 * for a < rows, b < cols.  The phase index is reduced exactly in 64-bit integers, the value computed in
 * double precision and stored as float2.
 */
OI_API int oi_twiddle(void* out, int rows, int cols, long long a0, long long b0, long long n, int sign, double scale,
                      void* stream);

/*
 * Band-limited forward spectrum (Scatter.py:10-35 restricted to a band):
 *   band[b][c][ir][ic] = scale * sum_{y,x} h[b][y][x][c] * wy[y][ir] * wx[x][ic]
 * with wx[x][ic] = exp(+2 pi i (m0c+ic) x / nx) and wy[y][ir] = exp(+2 pi i (m0r+ir) y / ny) (oi_twiddle).
 * scratch: float2 [batch * nch * ny * bc].
 */
OI_API int oi_band_spectrum(const void* field, int kind, int batch, int ny, int nx, int nch, int br, int bc,
                            const void* wx, const void* wy, float scale, void* scratch, void* band, void* stream);

/*
 * oi_band_spectrum without a scratch argument, for callers that cannot allocate device memory -- code handed
 * only the pointers of a host application that owns every allocation, or running inside a memory budget that
 * is already fully given out.  No counterpart in the reference (which allocates freely through torch).
 *   - Same inputs, output and result as oi_band_spectrum; the row-transform scratch is an array built into the
 *     library, OI_NOALLOC_SCRATCH_COMPLEX complex values (16 MiB) on every GPU that loads it, held until the
 *     process exits.  batch * nch * ny * bc above that capacity is rejected with OI_ERANGE.
 *   - Calls no cudaMalloc / cudaFree.  A call looks up the array's device address (cudaGetSymbolAddress) on
 *     the current device unless its stream is capturing, when it uses the address the previous call found; so
 *     make the first call on each device before any stream capture.
 *   - All calls on a device share the one array: calls that can overlap on the GPU (different streams without
 *     ordering between them) race.  Nothing in the array needs clearing between calls.
 */
#define OI_NOALLOC_SCRATCH_COMPLEX (1LL << 21) /* built-in scratch of oi_band_spectrum_noalloc, complex values */
OI_API int oi_band_spectrum_noalloc(const void* field, int kind, int batch, int ny, int nx, int nch, int br, int bc,
                                    const void* wx, const void* wy, float scale, void* band, void* stream);

/*
 * Abbe pupils (CalculateAerialImage.py:46-75), one per (plane z, source point j, field component e):
 *   pupil[z][j*ne+e][ir][ic] = valid * obliquity * exp(2 pi i W) * defocus_z * transfer_e     (complex64)
 *   weight[z][j*ne+e]        = index_image * v[j] / weight_sum
 * fr[ir] / fc[ic]: the reference's float32 row (Y, g) and column (X, f) frequency values of the band.
 * sx/sy/sv: float32 source points; focus: double [nz] (all device pointers).
 * zern (37 Fringe coefficients, may be NULL) and jones (Px.re, Px.im, Py.re, Py.im) are HOST pointers.
 * Membership `valid` repeats the reference's float32 test (CalculateAerialImage.py:43-57) bit for bit.
 */
OI_API int oi_abbe_pupils(const float* fr, const float* fc, int br, int bc, const float* sx, const float* sy,
                          const float* sv, int nsrc, double weight_sum, const double* focus, int nz, const double* zern,
                          int vector,
                          const double* jones, double na, double mag, double index_image, double wavelength,
                          void* pupil, float* weight, void* stream);

/*
 * oi_abbe_pupils with a Jones vector per source point: jones_pts is a DEVICE array [nsrc][4] of doubles (Px.re,
 * Px.im, Py.re, Py.im of point j), in place of the constant host `jones` -- a polarisation map (Source.py:183-221)
 * or one eigen-polarisation of a coherency matrix.  Scalar mode (vector = 0) does not read it.
 */
OI_API int oi_abbe_pupils_pol(const float* fr, const float* fc, int br, int bc, const float* sx, const float* sy,
                              const float* sv, int nsrc, double weight_sum, const double* focus, int nz,
                              const double* zern, int vector, const double* jones_pts, double na, double mag,
                              double index_image, double wavelength, void* pupil, float* weight, void* stream);

/*
 * Coherent sum on the coarse grid (the |.|^2 accumulation of both imaging paths):
 *   coarse[b][z][sr][sc] = sum_{k<nk, c<nch} w[z][k] |sum_{ir,ic} fr[sr][ir] (P[z][k] .* band[b][c])[ir][ic] fcs[ic][sc]|^2
 * fr  = oi_twiddle(mr x br, sign -1) row phases, fcs = oi_twiddle(bc x mc, sign -1) column phases.
 * mc must be a multiple of 64 and at most 256; br, bc at most 256.
 * `pupil_batch_stride` = 0 shares the pupils across the batch (SOCS kernels), else it is the element stride
 * between images' pupil sets.  The fields (k, c), f = k*nch + c, are split over `nsplit` partial sums:
 * f = s, s + nsplit, ... go to coarse[s][b][z][sr][sc] (float [nsplit][batch][nz][mr][mc]); the coarse-to-image
 * stage adds them with nparts = nsplit.
 */
OI_API int oi_coherent_coarse(const void* band, int batch, int nch, int br, int bc, const void* pupil,
                              long long pupil_batch_stride, const float* weight, int nz, int nk, int mr, int mc,
                              const void* frow, const void* fcol, int nsplit, float* coarse, void* stream);

/*
 * Exact band-limited resampling of the coarse intensity to the output grid:
 *   out[i][y][x] = sum_{|qr|<br, |qc|<bc} Ihat_i(q) exp(-2 pi i (qr y/ny + qc x/nx)),
 *   Ihat_i(q)    = 1/(mr mc) sum_s coarse[i][s] exp(+2 pi i (qr sr/mr + qc sc/mc)),
 * where coarse holds `nparts` partial sums one after another (count*mr*mc floats each; 1 for oi_coherent_coarse).
 * With nparts > 1 the partials are added into the first one in place (the buffer is scratch afterwards).
 * Tables (oi_twiddle): gc [mc][bc] (+, b0=0), gr [mr][2br-1] (+, b0=-(br-1)), sy [ny][2br-1] (-, b0=-(br-1)),
 * sx [bc][nx] (-, a0=0).  scratch: float2 [count * (2br-1) * bc].
 */
OI_API int oi_coarse_to_image(float* coarse, int nparts, int count, int mr, int mc, int br, int bc,
                              const void* gc, const void* gr, const void* sy, const void* sx, int ny, int nx,
                              void* scratch, float* out, void* stream);

/*
 * FFT form of the two N-point transforms (grids of 256, 512, 1024 or 2048 per axis).  oi_fft_supported(ny, nx)
 * returns 1 when both axes qualify.
 *
 * oi_band_spectrum_fft: as oi_band_spectrum for real float32 / uint8 masks [batch][ny][nx], band rows
 *   m0r .. m0r+br-1 and columns m0c .. m0c+bc-1 (2 max|m_c| < nx, br <= ny).  wn_x / wn_y: the FFT tables of
 *   n = nx / ny (n1 = n/32): oi_twiddle(32, n1, 0, 0, n, +1) followed by oi_twiddle(n1, n1, 0, 0, n1, +1) in one
 *   buffer.  scratch: float2 [batch * bc * ny].  band: float2 [batch][br][bc].
 * oi_coarse_to_image_fft: as oi_coarse_to_image (same gc, gr tables), with the y and x syntheses done as
 *   pruned inverse FFTs; the coarse input holds `nparts` partial sums one after another (count*mr*mc floats
 *   each).  When wm_r / wm_c (oi_twiddle(1, m, 1, 0, m, +1) for m = mr / mc) are given and mr, mc are 64 or
 *   128, the coarse spectrum is an FFT too (one block per image); else it is the DFT of oi_coarse_to_image.
 *   scratch_ihat: float2 [count * (2br-1) * bc]; scratch_v: float2 [count * bc * ny].
 */
OI_API int oi_fft_supported(int ny, int nx);
OI_API int oi_band_spectrum_fft(const void* field, int kind, int batch, int ny, int nx, int m0r, int br, int m0c,
                                int bc, const void* wn_x, const void* wn_y, float scale, void* scratch, void* band,
                                void* stream);
OI_API int oi_coarse_to_image_fft(float* coarse, int nparts, int count, int mr, int mc, int br, int bc,
                                  const void* gc, const void* gr, const void* wm_r, const void* wm_c,
                                  const void* wn_y, const void* wn_x, int ny, int nx, void* scratch_ihat,
                                  void* scratch_v, float* out, void* stream);

/*
 * FFT form of oi_coherent_coarse for coarse grids of 64 or 128 per axis, or of 256 x 256 (bands up to 128 x 128;
 * one block of 512 threads per SM holding its 256 x 256 partial sum in tensor memory): the fields of each
 * (image, plane) are split over `nsplit` blocks that write partial sums coarse[s][b][z][mr][mc] (s < nsplit), which
 * oi_coarse_to_image_fft adds (nparts = nsplit).  wr / wc: oi_twiddle(1, m, 1, 0, m, +1) for m = mr / mc.
 * The band starts at frequency (m0r, m0c).
 */
OI_API int oi_coherent_coarse_fft(const void* band, int batch, int nch, int m0r, int br, int m0c, int bc,
                                  const void* pupil, long long pupil_batch_stride, const float* weight, int nz,
                                  int nk, int mr, int mc, const void* wr, const void* wc, int nsplit, float* coarse,
                                  void* stream);

/*
 * Split-BF16x3 form of oi_coherent_coarse_fft on the 5th-generation tensor cores, coarse grid 128 x 128,
 * band at most 64 x 64.  Each real operand x is split into bf16 hi = bf16(x), lo = bf16(x - hi) and a product
 * is hi*hi + hi*lo + lo*hi accumulated in FP32 (about 16 significant bits).  Same arguments and result as
 * oi_coherent_coarse_fft, except that the work is cut by task: the batch*nz*nk*nch fields run as `ctas`
 * contiguous ranges and `coarse` holds `nparts` partial sums, [nparts][batch][nz][128][128], added in order
 * by oi_coarse_to_image(_fft) with the same nparts.  oi_coherent_tc_layout gives ctas (one per SM) and the
 * nparts that cut needs; a smaller nparts is OI_ERANGE.  `consts` is the band's constant operand image written
 * by oi_tc_constants (16-byte aligned).  A wait on the tensor pipe or a copy that exceeds 2 s ends the kernel
 * early and sets the device status (oi_device_status) to 1; the result is then invalid.
 */
OI_API int oi_coherent_tc_layout(long long images, int fields, int* ctas, int* nparts);
OI_API int oi_coherent_coarse_tc(const void* band, int batch, int nch, int m0r, int br, int m0c, int bc,
                                 const void* pupil, long long pupil_batch_stride, const float* weight, int nz,
                                 int nk, const void* consts, int ctas, int nparts, float* coarse, void* stream);

/*
 * The constant operand image of oi_coherent_coarse_tc for a band starting at (m0r, m0c): the split DFT
 * matrices exp(-2 pi i (m0+i) s / 128), s < 128, i < 64, in the kernel's swizzled shared-memory layout.
 * 98304 bytes when m0r == m0c, else 163840.  wr / wc: oi_twiddle(1, 128, 1, 0, 128, +1).
 */
OI_API int oi_tc_constants(int m0r, int m0c, const void* wr, const void* wc, void* image, long long bytes,
                           void* stream);

/*
 * The N-point row passes of the split-BF16x3 form on the tensor cores (dense DFT contractions, bf16 hi / lo
 * operands, FP32 accumulate).  Grids: ny a multiple of 128 (the row blocks), nx a multiple of 128 up to 4096;
 * band width bc <= 64.
 *   oi_rows_fwd_tc  t[b][ic][y] = sum_x field[b][y][x] exp(+2 pi i (m0c+ic) x / nx)  (float32 or uint8 masks;
 *                   t as the scratch of oi_band_spectrum_fft, float2 [batch][bc][ny])
 *   oi_rows_inv_tc  out[i][y][x] = sum_{qc<bc} Re(v[i][qc][y] exp(-2 pi i qc x / nx))  (v float2 [count][bc][ny];
 *                   vtiles: scratch of count * ny * 512 bytes that receives v as bf16 operand tiles)
 *   oi_rows_fwd_tc_half  the same for ic = 0 .. bch-1 at m0c = 0 (bch <= 32): the non-negative columns of a
 *                   real mask's row transform (t[-ic] = conj(t[ic])), t float2 [batch][bch][ny]
 * `consts` is the constant operand image from oi_rows_tc_constants: which = 0 (forward; depends on nx, m0c, bc;
 * nx/64 * 32768 bytes), 1 (inverse; depends on nx, bc; nx/128 * 65536 bytes) or 2 (forward half for
 * oi_rows_fwd_tc_half, given the symmetric band m0c = -(bc-1)/2, bc odd <= 63, it covers bch = (bc+1)/2 columns;
 * nx/64 * 16384 bytes).  A wait that exceeds 2 s ends the kernel early and sets the device status.
 * oi_band_spectrum_tc and oi_coarse_to_image_tc are oi_band_spectrum_fft and oi_coarse_to_image_fft (coarse grid
 * 128 x 128) with these row passes; oi_coarse_to_image_tc writes the column pass straight into the V operand tiles
 * (scratch_tiles, count * ny * 512 bytes; scratch_v is unused and may be NULL).
 */
OI_API int oi_rows_tc_constants(int which, int nx, int m0c, int bc, void* image, long long bytes, void* stream);
OI_API int oi_rows_fwd_tc(const void* field, int kind, int batch, int ny, int nx, int m0c, int bc,
                          const void* consts, void* t, void* stream);
OI_API int oi_rows_fwd_tc_half(const void* field, int kind, int batch, int ny, int nx, int bch, const void* consts,
                               void* t, void* stream);
OI_API int oi_rows_inv_tc(const void* v, int count, int ny, int nx, int bc, const void* consts, void* vtiles,
                          float* out, void* stream);
/* The synthesis row pass alone, from V operand tiles already written (by oi_rows_inv_tc's conversion or by the
 * column pass of oi_coarse_to_image_tc): the second half of oi_rows_inv_tc. */
OI_API int oi_rows_inv_tc_tiles(const void* vtiles, int count, int ny, int nx, const void* consts, float* out,
                                void* stream);
OI_API int oi_band_spectrum_tc(const void* field, int kind, int batch, int ny, int nx, int m0r, int br, int m0c,
                               int bc, const void* wconsts, const void* wn_y, float scale, void* scratch,
                               void* band, void* stream);
/* oi_band_spectrum_tc for a real mask and an odd symmetric band (m0r = -(br-1)/2, m0c = -(bc-1)/2, bc <= 63):
 * the row pass computes the band's (bc+1)/2 non-negative columns only (oi_rows_fwd_tc_half, hconsts from
 * oi_rows_tc_constants(2, nx, m0c, bc, ...)) and the column pass writes each column and its mirror
 * band[-ky][-kx] = conj(band[ky][kx]).  scratch: batch * ny * (bc+1)/2 complex.  Same band as
 * oi_band_spectrum_tc (Scatter.CalculateSpectrum, Scatter.py:10-35, restricted to the band). */
OI_API int oi_band_spectrum_tc_sym(const void* field, int kind, int batch, int ny, int nx, int br, int bc,
                                   const void* hconsts, const void* wn_y, float scale, void* scratch, void* band,
                                   void* stream);
OI_API int oi_coarse_to_image_tc(float* coarse, int nparts, int count, int br, int bc, const void* wm_r,
                                 const void* wm_c, const void* wn_y, const void* cconsts, int ny, int nx,
                                 void* scratch_ihat, void* scratch_v, void* scratch_tiles, float* out, void* stream);

/*
 * The coarse-to-image stage of the split-BF16x3 form with the coarse spectrum and the column synthesis on the
 * tensor cores as well (the final transform of CalculateAerialImage_SOCS.py:7-10 restricted to the intensity's
 * band): per image two real GEMMs,
 *   U[sr][n] = sum_sc c[sr][sc] G[sc][n]   G = ((qc ? 2 : 1)/128) (cos | sin)(2 pi qc sc / 128)  (n = re|im x qc < bc)
 *   v[y][n]  = sum_sr A[y][sr] U[sr][n]   A = (1/128) sum_{|qr| < br} cos(2 pi qr (sr/128 - y/ny))
 * c the coarse intensity (128 x 128, the sum of its nparts partial sums), v the band rows of the image spectrum
 * written as the V operand tiles of the row pass (oi_rows_inv_tc_tiles layout).  ny a multiple of 128 up to 4096,
 * bc <= 64, 2br-1 <= 128.
 *   oi_synth_tc_constants  the constant image of G and A for (ny, br, bc): (1 + ny/128) * 65536 bytes
 *   oi_synth_tiles_tc      V tiles [count * ny / 128][64 KB] from coarse [nparts][count][128][128]
 *   oi_coarse_to_image_tcs oi_synth_tiles_tc then oi_rows_inv_tc_tiles (cconsts from oi_rows_tc_constants(1, ...)):
 *                          the same result as oi_coarse_to_image_tc
 * A wait that exceeds 2 s ends the kernel early and sets the device status.
 */
OI_API int oi_synth_tc_constants(int ny, int br, int bc, void* image, long long bytes, void* stream);
OI_API int oi_synth_tiles_tc(const float* coarse, int nparts, int count, int br, int bc, const void* sconsts, int ny,
                             void* tiles, void* stream);
OI_API int oi_coarse_to_image_tcs(const float* coarse, int nparts, int count, int br, int bc, const void* sconsts,
                                  const void* cconsts, int ny, int nx, void* scratch_tiles, float* out, void* stream);

/* The device status word (0 = no error) set by kernels whose bounded waits expired; optionally cleared.
 * Synchronous (reads device memory). */
OI_API int oi_device_status(int* status, int reset);

/* The failure path of the tensor-core kernels' bounded waits, on its own (no counterpart in the reference): one
 * CTA allocates tmem_cols columns of tensor memory (a power of two, 32..512), waits with the kernels' bounded wait
 * -- limit_ns, at most 100 ms -- on a barrier that nothing completes, sets the device status to 1, releases the
 * tensor memory and returns.  For tests of the status reporting and of the context staying usable. */
OI_API int oi_wait_probe(long long limit_ns, int tmem_cols, void* stream);

/* Kernel launches this library has enqueued since it was loaded (launches captured into a CUDA graph are
 * counted once, at capture). */
OI_API int oi_launch_count(long long* count);


/*
 * The synthesis half of oi_coarse_to_image(_fft) on its own: a real image from the Hermitian half of its
 * spectrum, out[i][y][x] = sum_{|qr|<br, 0<=qc<bc} Re(ihat[i][qr+br-1][qc] exp(-2 pi i (qr y/ny + qc x/nx))),
 * with the qc > 0 terms already doubled by the caller.  DFT form: sy [ny][2br-1] (-, b0=-(br-1)) and
 * sx [bc][nx] tables of oi_coarse_to_image.  FFT form: wn tables as oi_coarse_to_image_fft, power-of-two grids,
 * scratch_v float2 [count * bc * ny].  Used by the adjoint (gradients) and for band-limited resampling.
 */
OI_API int oi_spectrum_to_image(const void* ihat, int count, int br, int bc, const void* sy, const void* sx, int ny,
                                int nx, float* out, void* stream);
OI_API int oi_spectrum_to_image_fft(const void* ihat, int count, int br, int bc, const void* wn_y, const void* wn_x,
                                    int ny, int nx, void* scratch_v, float* out, void* stream);
/*
 * The input of oi_spectrum_to_image_fft from a coarse intensity held as nparts partial sums ([nparts][count][mr][mc]
 * float32, oi_coherent_coarse_fft's output on a 256 x 256 or larger power-of-two coarse grid):
 * ihat[i][qr+br-1][qc] = w(qc) / (mr mc) sum_{y,x} (sum_p coarse[p][i][y][x]) exp(+2 pi i (qr y/mr + qc x/mc)),
 * |qr| < br, 0 <= qc < bc, w(0) = 1, w(qc > 0) = 2.  wn_c / wn_r: the FFT tables of mc and mr (as wn_x / wn_y of
 * oi_band_spectrum_fft); scratch: count * mr * bc complex.  The parts are summed as the row pass loads them.
 */
OI_API int oi_coarse_half_spectrum_fft(const float* coarse, int nparts, int count, int mr, int mc, int br, int bc,
                                       const void* wn_c, const void* wn_r, void* scratch, void* ihat, void* stream);

/*
 * Adjoint of the coherent sum (inverse lithography; no counterpart in the reference, whose gradients come from
 * torch autograd through its FFTs).  For fields A_f = P[z][k] .* band[b][c] and the band-limited coarse copy
 * gcoarse[b][z] (mr x mc = 128 x 128) of dL/dI:
 *   wout[s][b][z][c][ir][ic] = sum_{f in split s} w[z][k] conj(P[z][k][ir][ic]) F_f(ir, ic),
 *   F_f(m) = sum_sr,sc gcoarse(s) E_f^c(s) exp(+2 pi i m.s/M)       (E_f^c: the field on the coarse grid),
 *   field_dot[b][z][f] = sum_s gcoarse(s) |E_f^c(s)|^2              (optional, NULL to skip).
 * The mask gradient is 2/(ny nx) Re sum_m W(m) exp(-2 pi i m.y/N) with W summed over s and z.  Band at most
 * 64 x 64 (2br-1, 2bc-1 <= 128); wr / wc: oi_twiddle(1, 128, 1, 0, 128, +1).
 */
OI_API int oi_coherent_adjoint(const void* band, int batch, int nch, int m0r, int br, int m0c, int bc,
                               const void* pupil, const float* weight, int nz, int nk, const float* gcoarse, int mr,
                               int mc, const void* wr, const void* wc, int nsplit, void* wout, float* field_dot,
                               void* stream);

/*
 * Shifted pupil matrix of the TCC (CalculateTCCMatrix.py:17-51), FP64, scaled for a Gram product:
 *   h[e][p][j] = sqrt(index_image * v[j] / weight_sum) * valid * obliquity * exp(2 pi i W) * defocus * transfer_e
 * p = i_f * lg + i_g over the TCC grid (ff = f32 row frequencies, gg = f32 column frequencies); ne = 1 or 3.
 * Membership repeats the reference's float32 test sqrt(f^2+g^2) <= 1 (CalculateTCCMatrix.py:27-29).
 * zern and jones are HOST pointers, as for oi_abbe_pupils.
 */
OI_API int oi_tcc_pupils64(const float* ff, int lf, const float* gg, int lg, const float* sx, const float* sy,
                           const float* sv, int nsrc, double weight_sum, double focus, const double* zern, int vector,
                           const double* jones, double na, double mag, double index_image, double wavelength,
                           void* h, void* stream);

/* oi_tcc_pupils64 with a Jones vector per source point (jones_pts: DEVICE [nsrc][4] doubles, as for
 * oi_abbe_pupils_pol; CalculateTCCMatrix.py:40-46 with Calc_PolarizationMap, Source.py:183-221). */
OI_API int oi_tcc_pupils64_pol(const float* ff, int lf, const float* gg, int lg, const float* sx, const float* sy,
                               const float* sv, int nsrc, double weight_sum, double focus, const double* zern,
                               int vector, const double* jones_pts, double na, double mag, double index_image,
                               double wavelength, void* h, void* stream);

/*
 * The k leading eigenpairs of the TCC in FP64 (DecomposeTCC_SOCS.py:7-9, where the reference runs a full
 * torch.svd of its complex64 TCC): block subspace iteration on p vectors with Cholesky-QR orthonormalisation and
 * Rayleigh-Ritz every 4 iterations (one-CTA Jacobi on the p x p projection), until the leading k residuals
 * ||T u - lambda u|| are below tol * lambda_0 or max_iter iterations have run.  The TCC is given densely (tcc:
 * complex128 [n][n], h NULL) or as its pupil factor (h: complex128 [ne][n][s] with TCC = sum_e h_e h_e^H,
 * tcc NULL; the TCC is not formed).  k <= p <= min(n, 64), p even.  Output: vecs complex128 [n][k] (row-major,
 * column i the eigenvector of vals[i]), vals double [k] descending, clamped at zero (device pointers); *iters
 * (host) the iterations run, negative when tol was not reached.  work: oi_eig_topk64_workspace bytes.  Unlike
 * the imaging entry points this one synchronises its stream (it reads the residuals to decide when to stop).
 */
OI_API int oi_eig_topk64_workspace(int n, int p, int ne, int s, long long* bytes);
OI_API int oi_eig_topk64(const void* tcc, const void* h, int ne, int n, int s, int k, int p, int max_iter, double tol,
                         void* vecs, double* vals, void* work, long long work_bytes, int* iters, void* stream);

/*
 * TCC = sum_e h_e h_e^H (GetTCCMatrix, CalculateTCCMatrix.py:58-75), complex128 [fg][fg], full Hermitian.
 */
OI_API int oi_tcc_assemble64(const void* h, int ne, int fg, int nsrc, void* tcc, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* OI_B200_H */
