// Lattice structure factor: StructureFactor::compute_structure_factor
// (src/sf/sf.cpp:85-285, lattice branch :164-246), FP64, one thread per q-point.
//
// Per axis with theta = l . q' (q' = R q) the Dirichlet kernel
//   S = pow(e^{i theta}, (1-N)/2) * (1 - pow(e^{i theta}, N)) / (1 - e^{i theta}),  S = N when
//   |1 - e^{i theta}| <= machine epsilon (component-wise, sf.cpp:203-208),
// with std::pow's principal branch; the b axis reproduces the reference as written
// (sf.cpp:212: lb[2]*lb[2] where lb[2]*q'z is meant, exp(i N theta_b) instead of pow); the
// result is e^{i q'.center} Sa Sb Sc.  The GPU class of the reference multiplies a basis
// factor (1 + e^{i q.t}) that its CPU class does not (src/sf/gpu/sf_gpu.cu:290-291); the CPU
// class is followed here.
#include <cuda_runtime.h>
#include <float.h>

#include <string>

#include "ana_sf.cuh"
#include "ana_sf_f32.cuh"
#include "cplx.cuh"
#include "hgx_internal.cuh"

namespace hgx {

struct SfArgs {
  SfLat L;
  Rot9d R;
  const double* qx;
  const double* qy;
  const double2* qz;
  int nqy, nqz;
  void* out;
};

template <typename OUT>
__global__ void __launch_bounds__(128) sf_lattice_kernel(SfArgs a) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nqz) return;
  long j = i % a.nqy;
  zd m[3];
  rotate_q(a.R, a.qx[j], a.qy[j], zd(a.qz[i]), m);
  const zd v = sf_lattice_eval(a.L, m);
  if (sizeof(OUT) == sizeof(double2))
    reinterpret_cast<double2*>(a.out)[i] = v.d2();
  else
    reinterpret_cast<float2*>(a.out)[i] = make_float2((float)v.x, (float)v.y);
}

// FP32C for a grid with real qz (ana_sf_f32.cuh: FP64 phase reduction, FP32 sines).
template <typename OUT>
__global__ void __launch_bounds__(128) sf_lattice_f32c_kernel(SfArgs a) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nqz) return;
  long j = i % a.nqy;
  const double qx = a.qx[j], qy = a.qy[j], qz = a.qz[i].x;
  double m[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) m[k] = a.R.r[3 * k] * qx + a.R.r[3 * k + 1] * qy + a.R.r[3 * k + 2] * qz;
  const cf v = sf_lattice_f32c(a.L, m);
  if (sizeof(OUT) == sizeof(double2))
    reinterpret_cast<double2*>(a.out)[i] = make_double2((double)v.x, (double)v.y);
  else
    reinterpret_cast<float2*>(a.out)[i] = make_float2(v.x, v.y);
}

}  // namespace hgx

using namespace hgx;

namespace hgx {

// Lattice::construct_vectors, src/model/structure.cpp:86-182 (ca = 1, gamma = 0 as the
// reference's Lattice constructor sets them).  type: LatticeType (include/common/enums.hpp:56-65).
// False for an unknown type or an hkl the type has no vectors for.
bool lattice_table(int type, const std::string& h, double* abc9, double* t3) {
  const double sqrt3 = sqrt(3.0);
  double a[3] = {0}, b[3] = {0}, c[3] = {0}, t[3] = {0};
  auto set = [](double* v, double x, double y, double z) { v[0] = x; v[1] = y; v[2] = z; };
  switch (type) {
    case 3:  // cubic
      if (h == "100") { set(a, 1, 0, 0); set(b, 0, 1, 0); set(c, 0, 0, 1); }
      else if (h == "110") { set(a, 1, 0, 0); set(b, 0., 1.4142, 0); set(c, 0., 0.7071, 0.7071); }
      else return false;
      break;
    case 2:  // bcc
      if (h == "100") { set(a, 1., 0., 0.); set(b, 0., 1., 0.); set(c, 0.5, 0.5, 0.5); }
      else if (h == "110") { set(a, 1.0, 0.0, 0); set(b, 0.5, 0.7071, 0); set(c, 0.0, 0.7071, 0.7071); }
      else return false;
      break;
    case 4:  // fcc
      if (h == "100") { set(a, 0.0, 0.5, 0.5); set(b, 0.5, 0.0, 0.5); set(c, 0.5, 0.5, 0.0); }
      else if (h == "111") { set(a, 1., 0., 0); set(b, 0.5, 0.866, -0.); set(c, 1., 0.5773, 0.866); }
      else return false;
      break;
    case 5:  // fco
      set(a, 1, 0, 0); set(b, 0.5, tan(0.0) / 2.0, 0); set(c, 0, 0, 1.0); set(t, 0.5, 0, 0.5);
      break;
    case 6:  // hcp
      set(a, 1, 0, 0); set(b, 0.5, 0.866, 0); set(c, 0.5, 0.2887, 0.8165);
      break;
    case 7:  // hex
      set(a, 1, 0, 0); set(b, 0.5, sqrt3 / 2.0, 0); set(c, 0, 0, 1);
      break;
    default:
      return false;
  }
  for (int i = 0; i < 3; ++i) {
    abc9[i] = a[i];
    abc9[3 + i] = b[i];
    abc9[6 + i] = c[i];
    if (t3) t3[i] = t[i];
  }
  return true;
}

}  // namespace hgx

extern "C" {

int hgx_lattice_vectors(int type, const char* hkl, double* abc9, double* t3) {
  if (!abc9) return fail(HGX_ERR_INVALID_ARG, "hgx_lattice_vectors: null output");
  if (type < 2 || type > 7) return fail(HGX_ERR_INVALID_ARG, "hgx_lattice_vectors: unknown lattice type");
  if (!lattice_table(type, hkl ? hkl : "100", abc9, t3))
    return fail(HGX_ERR_INVALID_ARG, "hgx_lattice_vectors: invalid lattice type and hkl");
  return HGX_OK;
}

int hgx_sf_lattice_ex(hgx_ctx c, hgx_qgrid g, const double* abc9, const double* repet,
                      const double* scaling, const double* center, const double* rot9, void* sf,
                      int sf_type, int precision) {
  if (precision != HGX_F64 && precision != HGX_F32C)
    return fail(HGX_ERR_INVALID_ARG, "hgx_sf_lattice: unknown precision");
  if (!c || !g || !abc9 || !repet || !scaling || !sf)
    return fail(HGX_ERR_INVALID_ARG, "hgx_sf_lattice: null argument");
  if (g->ctx != c) return fail(HGX_ERR_INVALID_ARG, "hgx_sf_lattice: grid of another context");
  if (sf_type != HGX_C128 && sf_type != HGX_C64)
    return fail(HGX_ERR_INVALID_ARG, "hgx_sf_lattice: unknown output type");
  SfArgs a;
  for (int i = 0; i < 3; ++i) {
    a.L.la[i] = abc9[i] * scaling[0];
    a.L.lb[i] = abc9[3 + i] * scaling[1];
    a.L.lc[i] = abc9[6 + i] * scaling[2];
    a.L.rep[i] = repet[i] < 1 ? 1 : repet[i];  // sf.cpp:164-166
    a.L.center[i] = center ? center[i] : 0.0;
  }
  static const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 9; ++i) a.R.r[i] = rot9 ? rot9[i] : eye[i];
  a.qx = g->qx;
  a.qy = g->qy;
  a.qz = g->qz;
  a.nqy = g->nqy;
  a.nqz = g->nqz;
  HGX_CUDA(cudaSetDevice(c->device));
  const size_t bytes = (sf_type == HGX_C64 ? sizeof(float2) : sizeof(double2)) * (size_t)g->nqz;
  DevBuf tmp;
  void* dout = nullptr;
  HGX_TRY(stage_out(c, sf, bytes, tmp, &dout));
  a.out = dout;
  dim3 grid((g->nqz + 127) / 128);
  bool integral = true;  // FP32C takes the closed form for integer repetitions
  for (int i = 0; i < 3; ++i) integral = integral && a.L.rep[i] == rint(a.L.rep[i]);
  if (precision == HGX_F32C && g->mode == 1 && integral) {
    if (sf_type == HGX_C64) sf_lattice_f32c_kernel<float2><<<grid, 128, 0, c->stream>>>(a);
    else sf_lattice_f32c_kernel<double2><<<grid, 128, 0, c->stream>>>(a);
  } else if (sf_type == HGX_C64) {
    sf_lattice_kernel<float2><<<grid, 128, 0, c->stream>>>(a);
  } else {
    sf_lattice_kernel<double2><<<grid, 128, 0, c->stream>>>(a);
  }
  HGX_CUDA(cudaGetLastError());
  return finish_out(c, sf, bytes, dout);
}

int hgx_sf_lattice(hgx_ctx c, hgx_qgrid g, const double* abc9, const double* repet,
                   const double* scaling, const double* center, const double* rot9, void* sf,
                   int sf_type) {
  return hgx_sf_lattice_ex(c, g, abc9, repet, scaling, center, rot9, sf, sf_type, HGX_F64);
}

}  // extern "C"
