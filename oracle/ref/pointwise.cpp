// C entry points over the reference's own pointwise functions, compiled from
// the reference tree unmodified (include/azeban/equations/
// incompressible_euler_functions.hpp, spectral_viscosity.hpp,
// include/azeban/operations/copy_to_padded_functions.hpp, complex.hpp), with
// the stand-ins of oracle/ref for the absent ZisaCore, ZisaMemory and fmt
// headers and for the CMake-generated config.hpp (double precision).
//
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref by oracle/build_ref.sh and
// used by tests/test_oracle_ref.py to pin the numpy oracle's pointwise stages
// against the reference's code.  The per-mode loops below follow the
// reference's CPU glue (include/azeban/equations/incompressible_euler.hpp
// :168-213 for computeB, :230-347 for computeDudt); the arithmetic they call
// is the reference's.
#include <azeban/config.hpp>
#include <azeban/equations/incompressible_euler_functions.hpp>
#include <azeban/equations/spectral_viscosity.hpp>
#include <azeban/operations/copy_to_padded_functions.hpp>

#include <cmath>

using azeban::complex_t;
using azeban::real_t;

namespace {

// nu(|k|) of one viscosity law, through the reference's eval().
real_t visc_eval(int type, double eps, double s, double k0, long long N, real_t k) {
  switch (type) {
    case 1: return azeban::SmoothCutoff1D(eps, s, k0).eval(k);
    case 2: return azeban::Step1D(eps, s, k0).eval(k);
    case 3: return azeban::Quadratic(eps, zisa::int_t(N)).eval(k);
    default: return azeban::NoViscosity().eval(k);
  }
}

}  // namespace

extern "C" {

// The scaling of computeB, 1 / (N^{d/2} M^{d/2}) (incompressible_euler.hpp:171-173).
double azref_norm(int dim, long long N, long long M) {
  const real_t n = real_t(N), m = real_t(M);
  if (dim == 2) return 1.0 / (zisa::pow<2>(zisa::sqrt(n)) * zisa::pow<2>(zisa::sqrt(m)));
  return 1.0 / (zisa::pow<3>(zisa::sqrt(n)) * zisa::pow<3>(zisa::sqrt(m)));
}

// B = products of norm * u in the reference's order, per point
// (incompressible_euler.hpp:168-213): u is [dim][n], B is [dim(dim+1)/2][n].
void azref_compute_B(int dim, long long n, double norm, const double *u, double *B) {
  for (long long i = 0; i < n; ++i) {
    if (dim == 2) {
      const real_t u1 = norm * u[i];
      const real_t u2 = norm * u[n + i];
      azeban::incompressible_euler_2d_compute_B(n, i, u1, u2, B);
    } else {
      const real_t u1 = norm * u[i];
      const real_t u2 = norm * u[n + i];
      const real_t u3 = norm * u[2 * n + i];
      azeban::incompressible_euler_3d_compute_B(n, i, u1, u2, u3, B);
    }
  }
}

// The per-mode right-hand side of the reference's CPU path for a list of
// modes (incompressible_euler.hpp:230-347, no forcing): signed indices
// idx[dim][n], B_hat[dim(dim+1)/2][n] and u_hat[dim][n] interleaved complex,
// dudt[dim][n] out.
void azref_dudt_modes(int dim, long long n, const int *idx, const double *B_hat, const double *u_hat,
                      int visc_type, double eps, double s, double k0, long long visc_N, double *dudt) {
  const complex_t *B = reinterpret_cast<const complex_t *>(B_hat);
  const complex_t *u = reinterpret_cast<const complex_t *>(u_hat);
  complex_t *out = reinterpret_cast<complex_t *>(dudt);
  const complex_t zero(0, 0);
  for (long long m = 0; m < n; ++m) {
    if (dim == 2) {
      const real_t k1 = 2 * zisa::pi * idx[m];
      const real_t k2 = 2 * zisa::pi * idx[n + m];
      const real_t absk2 = k1 * k1 + k2 * k2;
      complex_t L1, L2;
      azeban::incompressible_euler_2d_compute_L(k1, k2, absk2, n, m, B, zero, zero, &L1, &L2);
      const real_t nu = visc_eval(visc_type, eps, s, k0, visc_N, zisa::sqrt(absk2));
      out[m] = absk2 == 0 ? complex_t(0) : -L1 + nu * u[m];
      out[n + m] = absk2 == 0 ? complex_t(0) : -L2 + nu * u[n + m];
    } else {
      const real_t k1 = 2 * zisa::pi * idx[m];
      const real_t k2 = 2 * zisa::pi * idx[n + m];
      const real_t k3 = 2 * zisa::pi * idx[2 * n + m];
      const real_t absk2 = k1 * k1 + k2 * k2 + k3 * k3;
      complex_t L1, L2, L3;
      azeban::incompressible_euler_3d_compute_L(k1, k2, k3, absk2, n, m, B, zero, zero, zero, &L1, &L2, &L3);
      const real_t nu = visc_eval(visc_type, eps, s, k0, visc_N, zisa::sqrt(absk2));
      out[m] = absk2 == 0 ? complex_t(0) : -L1 + nu * u[m];
      out[n + m] = absk2 == 0 ? complex_t(0) : -L2 + nu * u[n + m];
      out[2 * n + m] = absk2 == 0 ? complex_t(0) : -L3 + nu * u[2 * n + m];
    }
  }
}

// nu(k) of one law for n wavenumber magnitudes.
void azref_visc_eval(int type, double eps, double s, double k0, long long N, long long n, const double *k,
                     double *out) {
  for (long long i = 0; i < n; ++i) out[i] = visc_eval(type, eps, s, k0, N, k[i]);
}

// Source index of destination index i along a full (compact == 0) or the
// compact last (compact == 1) axis padded from src_n to dst_n, or -1 where
// the reference writes the pad value (copy_to_padded_functions.hpp:9-63).
long long azref_pad_index(int compact, long long src_n, long long dst_n, long long i) {
  complex_t cell(0, 0);
  zisa::array_view<complex_t, 1> dst{&cell};
  unsigned long i_src = 0;
  const bool padded =
      compact ? azeban::pad_dim<true, true, 1>(dst, 0, src_n, dst_n, i, complex_t(0), &i_src)
              : azeban::pad_dim<true, false, 1>(dst, 0, src_n, dst_n, i, complex_t(0), &i_src);
  return padded ? -1 : (long long)i_src;
}

}  // extern "C"
