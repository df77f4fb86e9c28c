// Pupil synthesis for both imaging paths, FP64 arithmetic.
//
// Abbe (CalculateAerialImage.py:46-75): for every focus plane z, source point j and field component e, the
// shifted pupil over the band:  valid * obliquity * exp(2 pi i W_zernike) * defocus_z * transfer_e.
// TCC  (CalculateTCCMatrix.py:17-51): the same shifted pupil on the TCC grid, as the matrix h[e][p][j]
// scaled by sqrt(n w_j / sum w), so that TCC = sum_e h_e h_e^H.
//
// Which samples lie inside the pupil is decided exactly as the reference decides it -- float32 arithmetic in
// the reference's operation order, with FMA contraction suppressed (__fmul_rn/__fadd_rn) -- because a sample
// on the edge that flips changes the image.  Everything after that is double precision.
#include "oi_common.cuh"

namespace oi {

struct Optics {
  double na, mag, index_image, wavelength;
  double pxr, pxi, pyr, pyi;  // Jones vector
  int vector;
  int has_zern;
  double zern[37];  // Fringe coefficients, passed by value with the launch
};

// Fringe Zernike Z1..Z37 in waves at (rho, theta) (Projection.py:13-128).
__device__ double fringe_zernike(const double* z, double r, double th) {
  double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4, r9 = r8 * r,
         r10 = r5 * r5, r12 = r6 * r6;
  double s1, c1, s2, c2, s3, c3, s4, c4, s5, c5;
  sincos(th, &s1, &c1);
  sincos(2 * th, &s2, &c2);
  sincos(3 * th, &s3, &c3);
  sincos(4 * th, &s4, &c4);
  sincos(5 * th, &s5, &c5);
  double a = z[0];
  a += z[1] * r * c1 + z[2] * r * s1 + z[3] * (2 * r2 - 1);
  a += z[4] * r2 * c2 + z[5] * r2 * s2;
  double p = 3 * r3 - 2 * r;
  a += z[6] * p * c1 + z[7] * p * s1 + z[8] * (6 * r4 - 6 * r2 + 1);
  a += z[9] * r3 * c3 + z[10] * r3 * s3;
  p = 4 * r4 - 3 * r2;
  a += z[11] * p * c2 + z[12] * p * s2;
  p = 10 * r5 - 12 * r3 + 3 * r;
  a += z[13] * p * c1 + z[14] * p * s1 + z[15] * (20 * r6 - 30 * r4 + 12 * r2 - 1);
  a += z[16] * r4 * c4 + z[17] * r4 * s4;
  p = 5 * r5 - 4 * r3;
  a += z[18] * p * c3 + z[19] * p * s3;
  p = 15 * r6 - 20 * r4 + 6 * r2;
  a += z[20] * p * c2 + z[21] * p * s2;
  p = 35 * r7 - 60 * r5 + 30 * r3 - 4 * r;
  a += z[22] * p * c1 + z[23] * p * s1 + z[24] * (70 * r8 - 140 * r6 + 90 * r4 - 20 * r2 + 1);
  a += z[25] * r5 * c5 + z[26] * r5 * s5;
  p = 6 * r6 - 5 * r4;
  a += z[27] * p * c4 + z[28] * p * s4;
  p = 21 * r7 - 30 * r5 + 10 * r3;
  a += z[29] * p * c3 + z[30] * p * s3;
  p = 56 * r8 - 105 * r6 + 60 * r4 - 10 * r2;
  a += z[31] * p * c2 + z[32] * p * s2;
  p = 126 * r9 - 280 * r7 + 210 * r5 - 60 * r3 + 5 * r;
  a += z[33] * p * c1 + z[34] * p * s1;
  a += z[35] * (252 * r10 - 630 * r8 + 560 * r6 - 210 * r4 + 30 * r2 - 1);
  a += z[36] * (924 * r12 - 2772 * r10 + 3150 * r8 - 1680 * r6 + 420 * r4 - 42 * r2 + 1);
  return a;
}

// Scalar pupil at shifted frequency (f, g) and focus z:  obliquity * exp(2 pi i W) * defocus.
// NaN where the reference yields NaN (obliquity or defocus root of a negative number).
__device__ double2 scalar_pupil(const Optics& o, double f, double g, double z) {
  double r2 = f * f + g * g;
  double k2 = (o.na / o.mag) * (o.na / o.mag);
  double obl = pow((1.0 - k2 * r2) / (1.0 - o.na * o.na * r2), 0.25);
  double ph = 2.0 * M_PI / o.wavelength * sqrt(o.index_image * o.index_image - k2 * r2) * z;
  if (o.has_zern) ph += 2.0 * M_PI * fringe_zernike(o.zern, sqrt(r2), atan2(g, f));
  double s, c;
  sincos(ph, &s, &c);
  return make_double2(obl * c, obl * s);
}

__device__ __forceinline__ double2 cdiv_real_den(double2 num, double2 den) {
  double d = den.x * den.x + den.y * den.y;
  return make_double2((num.x * den.x + num.y * den.y) / d, (num.y * den.x - num.x * den.y) / d);
}

// The Jones vector of source point j: per point from `jones_pts` (device, [nsrc][4] doubles: Px.re, Px.im,
// Py.re, Py.im -- a polarisation map, Source.py:183-221) when given, else the constant one of the optics
// (PolarizationVector, Source.py:222-226).
__device__ __forceinline__ void jones_of(const Optics& o, const double* __restrict__ jones_pts, int j, double2& px,
                                         double2& py) {
  if (jones_pts) {
    const double* q = jones_pts + 4 * (long long)j;
    px = make_double2(q[0], q[1]);
    py = make_double2(q[2], q[3]);
  } else {
    px = make_double2(o.pxr, o.pxi);
    py = make_double2(o.pyr, o.pyi);
  }
}

// Polarisation transfer (CalculateCharacteristicMatrix.py:3-17 applied to the Jones vector (px, py),
// CalculateAerialImage.py:72-74): component e of (Px M0x? + Py M0y?).
__device__ void transfer(const Optics& o, double f, double g, double2 px, double2 py, double2 out[3]) {
  double al = o.na / o.index_image * f, be = o.na / o.index_image * g;
  double d = 1.0 - al * al - be * be;
  double2 gam = d >= 0 ? make_double2(sqrt(d), 0.0) : make_double2(0.0, sqrt(-d));
  double2 onepg = make_double2(1.0 + gam.x, gam.y);
  double2 mxx = cdiv_real_den(make_double2(al * al, 0.0), onepg);
  mxx = make_double2(1.0 - mxx.x, -mxx.y);
  double2 myx = cdiv_real_den(make_double2(-al * be, 0.0), onepg);
  double2 myy = cdiv_real_den(make_double2(be * be, 0.0), onepg);
  myy = make_double2(1.0 - myy.x, -myy.y);
  double2 t0 = cmul(px, mxx), t1 = cmul(py, myx);
  out[0] = make_double2(t0.x + t1.x, t0.y + t1.y);
  t0 = cmul(px, myx);
  t1 = cmul(py, myy);
  out[1] = make_double2(t0.x + t1.x, t0.y + t1.y);
  out[2] = make_double2(-(px.x * al + py.x * be), -(px.y * al + py.y * be));
}

// grid over (ir, ic) x j x z; each thread writes all ne components of one sample.
__global__ void abbe_pupil_kernel(Optics o, const float* __restrict__ fr, const float* __restrict__ fc, int br, int bc,
                                  const float* __restrict__ sx, const float* __restrict__ sy,
                                  const float* __restrict__ sv, int nsrc, const double* __restrict__ focus,
                                  double wnorm, const double* __restrict__ jones_pts, float2* __restrict__ pupil,
                                  float* __restrict__ weight) {
  const int ne = o.vector ? 3 : 1;
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, z = blockIdx.z;
  const long long plane = (long long)br * bc;
  if (idx == 0)
    for (int e = 0; e < ne; ++e) weight[((long long)z * nsrc + j) * ne + e] = (float)(wnorm * sv[j]);
  if (idx >= plane) return;
  const int ir = (int)(idx / bc), ic = (int)(idx % bc);
  const float fm = fr[ir], gm = fc[ic], X = sx[j], Y = sy[j];
  // float32 membership, CalculateAerialImage.py:43-57:  (fm^2+gm^2) + 2*(X fm + Y gm) + (X^2+Y^2) <= 1
  float fg2 = __fadd_rn(__fmul_rn(fm, fm), __fmul_rn(gm, gm));
  float t = __fadd_rn(__fmul_rn(X, fm), __fmul_rn(Y, gm));
  float xy2 = __fadd_rn(__fmul_rn(X, X), __fmul_rn(Y, Y));
  float rho2 = __fadd_rn(__fadd_rn(fg2, __fmul_rn(2.0f, t)), xy2);
  float2* out = pupil + (((long long)z * nsrc + j) * ne) * plane + idx;
  if (!(rho2 <= 1.0f)) {
    for (int e = 0; e < ne; ++e) out[e * plane] = make_float2(0.f, 0.f);
    return;
  }
  double f = (double)fm + (double)X, g = (double)gm + (double)Y;
  double2 p = scalar_pupil(o, f, g, focus[z]);
  if (!o.vector) {
    out[0] = make_float2((float)p.x, (float)p.y);
    return;
  }
  double2 tr[3], px, py;
  jones_of(o, jones_pts, j, px, py);
  transfer(o, f, g, px, py, tr);
  for (int e = 0; e < 3; ++e) {
    double2 v = cmul(p, tr[e]);
    out[e * plane] = make_float2((float)v.x, (float)v.y);
  }
}

// grid over p (TCC grid point) x j.  h[e][p][j].
__global__ void tcc_pupil_kernel(Optics o, const float* __restrict__ ff, int lf, const float* __restrict__ gg, int lg,
                                 const float* __restrict__ sx, const float* __restrict__ sy,
                                 const float* __restrict__ sv, int nsrc, double focus, double wnorm,
                                 const double* __restrict__ jones_pts, double2* __restrict__ h) {
  const int ne = o.vector ? 3 : 1;
  const long long fg = (long long)lf * lg;
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= fg * nsrc) return;
  const long long p = idx / nsrc;
  const int j = (int)(idx % nsrc);
  const int i_f = (int)(p / lg), i_g = (int)(p % lg);
  const float X = sx[j], Y = sy[j];
  // float32 membership, CalculateTCCMatrix.py:25-29:  sqrt((ff+X)^2 + (gg+Y)^2) <= 1
  float nf = __fadd_rn(ff[i_f], X), ng = __fadd_rn(gg[i_g], Y);
  float rho = __fsqrt_rn(__fadd_rn(__fmul_rn(nf, nf), __fmul_rn(ng, ng)));
  const long long plane = fg * nsrc;
  double2* out = h + idx;
  if (!(rho <= 1.0f)) {
    for (int e = 0; e < ne; ++e) out[e * plane] = make_double2(0.0, 0.0);
    return;
  }
  double f = (double)ff[i_f] + (double)X, g = (double)gg[i_g] + (double)Y;
  double2 pu = scalar_pupil(o, f, g, focus);
  double amp = sqrt(wnorm * (double)sv[j]);
  pu = make_double2(pu.x * amp, pu.y * amp);
  if (!o.vector) {
    out[0] = pu;
    return;
  }
  double2 tr[3], px, py;
  jones_of(o, jones_pts, j, px, py);
  transfer(o, f, g, px, py, tr);
  for (int e = 0; e < 3; ++e) out[e * plane] = cmul(pu, tr[e]);
}

static void set_optics(Optics& o, const double* zern, int vector, const double* jones, double na, double mag,
                       double index_image, double wavelength) {
  o.na = na;
  o.mag = mag;
  o.index_image = index_image;
  o.wavelength = wavelength;
  o.pxr = jones[0];
  o.pxi = jones[1];
  o.pyr = jones[2];
  o.pyi = jones[3];
  o.vector = vector ? 1 : 0;
  o.has_zern = 0;
  for (int i = 0; i < 37; ++i) {
    o.zern[i] = zern ? zern[i] : 0.0;
    if (o.zern[i] != 0.0) o.has_zern = 1;
  }
}

}  // namespace oi

namespace oi {

static int abbe_pupils(const float* fr, const float* fc, int br, int bc, const float* sx, const float* sy,
                       const float* sv, int nsrc, double weight_sum, const double* focus, int nz, const double* zern,
                       int vector, const double* jones, const double* jones_pts, double na, double mag,
                       double index_image, double wavelength, void* pupil, float* weight, void* stream,
                       const char* what) {
  if (!fr || !fc || !sx || !sy || !sv || !focus || (!jones && !jones_pts) || !pupil || !weight || br <= 0 ||
      bc <= 0 || nsrc <= 0 || nz <= 0)
    return fail(OI_EINVAL, "%s: bad arguments", what);
  if (nsrc > 65535 || nz > 65535) return fail(OI_ERANGE, "%s: too many source points or planes", what);
  cudaStream_t s = (cudaStream_t)stream;
  Optics o;
  const double none[4] = {1.0, 0.0, 0.0, 0.0};
  set_optics(o, zern, vector, jones ? jones : none, na, mag, index_image, wavelength);
  long long plane = (long long)br * bc;
  dim3 grid((unsigned)ceil_div(plane, 128), (unsigned)nsrc, (unsigned)nz);
  abbe_pupil_kernel<<<grid, 128, 0, s>>>(o, fr, fc, br, bc, sx, sy, sv, nsrc, focus, index_image / weight_sum,
                                         jones_pts, (float2*)pupil, weight);
  oi::note_launch();
  return check_launch(what);
}

static int tcc_pupils64(const float* ff, int lf, const float* gg, int lg, const float* sx, const float* sy,
                        const float* sv, int nsrc, double weight_sum, double focus, const double* zern, int vector,
                        const double* jones, const double* jones_pts, double na, double mag, double index_image,
                        double wavelength, void* h, void* stream, const char* what) {
  if (!ff || !gg || !sx || !sy || !sv || (!jones && !jones_pts) || !h || lf <= 0 || lg <= 0 || nsrc <= 0)
    return fail(OI_EINVAL, "%s: bad arguments", what);
  cudaStream_t s = (cudaStream_t)stream;
  Optics o;
  const double none[4] = {1.0, 0.0, 0.0, 0.0};
  set_optics(o, zern, vector, jones ? jones : none, na, mag, index_image, wavelength);
  long long total = (long long)lf * lg * nsrc;
  tcc_pupil_kernel<<<(unsigned)ceil_div(total, 128), 128, 0, s>>>(o, ff, lf, gg, lg, sx, sy, sv, nsrc, focus,
                                                                   index_image / weight_sum, jones_pts, (double2*)h);
  oi::note_launch();
  return check_launch(what);
}

}  // namespace oi

extern "C" int oi_abbe_pupils(const float* fr, const float* fc, int br, int bc, const float* sx, const float* sy,
                              const float* sv, int nsrc, double weight_sum, const double* focus, int nz,
                              const double* zern, int vector, const double* jones, double na, double mag,
                              double index_image, double wavelength, void* pupil, float* weight, void* stream) {
  if (!jones) return oi::fail(OI_EINVAL, "oi_abbe_pupils: bad arguments");
  return oi::abbe_pupils(fr, fc, br, bc, sx, sy, sv, nsrc, weight_sum, focus, nz, zern, vector, jones, nullptr, na,
                         mag, index_image, wavelength, pupil, weight, stream, "oi_abbe_pupils");
}

extern "C" int oi_abbe_pupils_pol(const float* fr, const float* fc, int br, int bc, const float* sx, const float* sy,
                                  const float* sv, int nsrc, double weight_sum, const double* focus, int nz,
                                  const double* zern, int vector, const double* jones_pts, double na, double mag,
                                  double index_image, double wavelength, void* pupil, float* weight, void* stream) {
  if (!jones_pts) return oi::fail(OI_EINVAL, "oi_abbe_pupils_pol: bad arguments");
  return oi::abbe_pupils(fr, fc, br, bc, sx, sy, sv, nsrc, weight_sum, focus, nz, zern, vector, nullptr, jones_pts,
                         na, mag, index_image, wavelength, pupil, weight, stream, "oi_abbe_pupils_pol");
}

extern "C" int oi_tcc_pupils64(const float* ff, int lf, const float* gg, int lg, const float* sx, const float* sy,
                               const float* sv, int nsrc, double weight_sum, double focus, const double* zern,
                               int vector, const double* jones, double na, double mag, double index_image,
                               double wavelength, void* h, void* stream) {
  if (!jones) return oi::fail(OI_EINVAL, "oi_tcc_pupils64: bad arguments");
  return oi::tcc_pupils64(ff, lf, gg, lg, sx, sy, sv, nsrc, weight_sum, focus, zern, vector, jones, nullptr, na, mag,
                          index_image, wavelength, h, stream, "oi_tcc_pupils64");
}

extern "C" int oi_tcc_pupils64_pol(const float* ff, int lf, const float* gg, int lg, const float* sx, const float* sy,
                                   const float* sv, int nsrc, double weight_sum, double focus, const double* zern,
                                   int vector, const double* jones_pts, double na, double mag, double index_image,
                                   double wavelength, void* h, void* stream) {
  if (!jones_pts) return oi::fail(OI_EINVAL, "oi_tcc_pupils64_pol: bad arguments");
  return oi::tcc_pupils64(ff, lf, gg, lg, sx, sy, sv, nsrc, weight_sum, focus, zern, vector, nullptr, jones_pts, na,
                          mag, index_image, wavelength, h, stream, "oi_tcc_pupils64_pol");
}
