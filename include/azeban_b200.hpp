/*
 * azeban_b200.hpp -- header-only C++ classes over the C ABI of
 * azeban_b200.h, with the signatures and semantics of azeban's own
 * interfaces for this path:
 *   azb::Equation<Dim>, azb::IncompressibleEuler<Dim>
 *       include/azeban/equations/equation.hpp:27-56,
 *       include/azeban/equations/incompressible_euler.hpp:39-124
 *   azb::TimeIntegrator<Dim>, azb::SSP_RK3<Dim>
 *       include/azeban/evolution/time_integrator.hpp:30-60, ssp_rk3.hpp:28-76
 *   azb::Simulation<Dim>    include/azeban/simulation.hpp:30-93, src/azeban/simulation.cpp:89-102
 *   azb::FFT<Dim>           include/azeban/operations/fft.hpp:37-121
 *   azb::Grid<Dim>          include/azeban/grid.hpp:30-53
 * Arrays are azb::array_view: the (shape, pointer, device) triple of zisa's
 * array_view, device memory in the reference's layouts.  Where azeban aborts
 * (LOG_ERR), these classes throw azb::Error carrying the library's status and
 * message.  dudt may be called in place; dt(C) is C / (N u_max) of the last
 * dudt with u_max the padded maximum over M^d, as the reference computes it.
 */
#ifndef AZEBAN_B200_HPP_
#define AZEBAN_B200_HPP_

#include <array>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "azeban_b200.h"

namespace azb {

class Error : public std::runtime_error {
 public:
  Error(az_status s, const std::string& where)
      : std::runtime_error(where + ": " + az_last_error_string()), status(s) {}
  az_status status;
};

inline void check(az_status s, const char* where) {
  if (s != AZ_OK) throw Error(s, where);
}

enum class device_type { cpu, cuda };

// (shape, pointer, device) of a non-owning view, as zisa::array_view.
template <typename T, int Rank>
struct array_view {
  std::array<std::size_t, Rank> shape_{};
  T* ptr_ = nullptr;
  device_type device_ = device_type::cuda;
  array_view() = default;
  array_view(const std::array<std::size_t, Rank>& shape, T* ptr, device_type dev = device_type::cuda)
      : shape_(shape), ptr_(ptr), device_(dev) {}
  T* raw() const { return ptr_; }
  std::size_t shape(int i) const { return shape_[i]; }
  std::size_t size() const {
    std::size_t n = 1;
    for (std::size_t s : shape_) n *= s;
    return n;
  }
  device_type memory_location() const { return device_; }
};

// Complex values are (re, im) pairs of the solve's precision.
template <typename Real>
struct Complex {
  Real x, y;
};

template <int Dim>
struct Grid {
  long long N_phys, N_phys_pad, N_fourier, N_fourier_pad;
  explicit Grid(long long N, long long M = 0)
      : N_phys(N), N_phys_pad(M ? M : 3 * N / 2), N_fourier(N / 2 + 1), N_fourier_pad((M ? M : 3 * N / 2) / 2 + 1) {}
  std::array<std::size_t, Dim + 1> shape_fourier(std::size_t n_vars) const {
    std::array<std::size_t, Dim + 1> s{};
    s[0] = n_vars;
    for (int d = 1; d < Dim; ++d) s[d] = std::size_t(N_phys);
    s[Dim] = std::size_t(N_fourier);
    return s;
  }
  std::array<std::size_t, Dim + 1> shape_phys(std::size_t n_vars) const {
    std::array<std::size_t, Dim + 1> s{};
    s[0] = n_vars;
    for (int d = 1; d <= Dim; ++d) s[d] = std::size_t(N_phys);
    return s;
  }
};

// The viscosity laws as the reference's factory leaves them
// (spectral_viscosity_factory.hpp:29-89): eps divided by N^{2s-1}, k0 = m0 N^theta.
struct SmoothCutoff1D {
  double eps, s, k0;
  az_visc c() const { return az_visc{AZ_VISC_SMOOTH_CUTOFF, eps, s, k0, 0}; }
};
struct Step1D {
  double eps, s, k0;
  az_visc c() const { return az_visc{AZ_VISC_STEP, eps, s, k0, 0}; }
};
struct Quadratic {
  double eps;
  long long N;
  az_visc c() const { return az_visc{AZ_VISC_QUADRATIC, eps, 0.0, 0.0, N}; }
};
struct NoViscosity {
  az_visc c() const { return az_visc{AZ_VISC_NONE, 0.0, 0.0, 0.0, 0}; }
};

// Equation<Dim> (equation.hpp:27-56) over spectral arrays of real type Real.
template <int Dim, typename Real = double>
class Equation {
 public:
  using complex_t = Complex<Real>;
  virtual ~Equation() = default;
  virtual void dudt(const array_view<complex_t, Dim + 1>& dudt_hat, const array_view<const complex_t, Dim + 1>& u_hat,
                    double t, double dt, double C) = 0;
  virtual double dt(double C) const = 0;
  virtual int n_vars() const = 0;
  virtual double visc() const = 0;
};

// IncompressibleEuler<Dim, Visc, NoForcing> (incompressible_euler.hpp:56-124),
// one member; Real double is the plain FP64 form, float the FP32-bulk form.
template <int Dim, typename Real = double>
class IncompressibleEuler final : public Equation<Dim, Real> {
 public:
  using complex_t = Complex<Real>;
  template <typename Visc>
  IncompressibleEuler(const Grid<Dim>& grid, const Visc& visc) : grid_(grid) {
    az_euler_desc d{};
    d.dim = Dim;
    d.N_phys = grid.N_phys;
    d.N_phys_pad = grid.N_phys_pad;
    d.precision = sizeof(Real) == 8 ? AZ_PREC_F64 : AZ_PREC_F32;
    d.visc = visc.c();
    d.batch = 1;
    check(az_euler_create(&d, &eq_), "IncompressibleEuler");
  }
  ~IncompressibleEuler() override { az_euler_destroy(eq_); }
  IncompressibleEuler(const IncompressibleEuler&) = delete;
  IncompressibleEuler& operator=(const IncompressibleEuler&) = delete;

  void dudt(const array_view<complex_t, Dim + 1>& dudt_hat, const array_view<const complex_t, Dim + 1>& u_hat,
            double t, double dt, double C) override {
    check_shape(dudt_hat.shape_);
    check_shape(u_hat.shape_);
    check(az_euler_dudt(eq_, dudt_hat.raw(), u_hat.raw(), t, dt, C, nullptr), "IncompressibleEuler::dudt");
  }
  double dt(double C) const override {
    double out = 0;
    check(az_euler_dt(eq_, C, nullptr, &out), "IncompressibleEuler::dt");
    return out;
  }
  int n_vars() const override { return Dim; }
  double visc() const override { return az_euler_visc(eq_); }
  const Grid<Dim>& grid() const { return grid_; }
  az_euler handle() const { return eq_; }

 private:
  void check_shape(const std::array<std::size_t, Dim + 1>& s) const {
    if (s != grid_.shape_fourier(Dim)) throw Error(AZ_ERR_INVALID, "IncompressibleEuler: wrong array shape");
  }
  Grid<Dim> grid_;
  az_euler eq_ = nullptr;
};

// TimeIntegrator<Dim> (time_integrator.hpp:30-60).
template <int Dim, typename Real = double>
class TimeIntegrator {
 public:
  using complex_t = Complex<Real>;
  virtual ~TimeIntegrator() = default;
  virtual double integrate(double t, double max_dt, double C, const array_view<complex_t, Dim + 1>& u) = 0;
};

// SSP_RK3<Dim> (ssp_rk3.hpp:28-64): one step in place, returns dt.
template <int Dim, typename Real = double>
class SSP_RK3 final : public TimeIntegrator<Dim, Real> {
 public:
  using complex_t = Complex<Real>;
  explicit SSP_RK3(const std::shared_ptr<IncompressibleEuler<Dim, Real>>& equation) : equation_(equation) {
    check(az_rk3_create(equation->handle(), &ts_), "SSP_RK3");
  }
  ~SSP_RK3() override { az_rk3_destroy(ts_); }
  SSP_RK3(const SSP_RK3&) = delete;
  SSP_RK3& operator=(const SSP_RK3&) = delete;
  double integrate(double t, double max_dt, double C, const array_view<complex_t, Dim + 1>& u) override {
    double dt = 0;
    check(az_rk3_integrate(ts_, t, max_dt, C, u.raw(), nullptr, &dt), "SSP_RK3::integrate");
    return dt;
  }
  az_rk3 handle() const { return ts_; }
  const std::shared_ptr<IncompressibleEuler<Dim, Real>>& equation() const { return equation_; }

 private:
  std::shared_ptr<IncompressibleEuler<Dim, Real>> equation_;
  az_rk3 ts_ = nullptr;
};

// Simulation<Dim> (simulation.cpp:89-102): owns the state; the step size and
// clock stay on the device.
template <int Dim, typename Real = double>
class Simulation {
 public:
  using complex_t = Complex<Real>;
  Simulation(const Grid<Dim>& grid, double C, const std::shared_ptr<SSP_RK3<Dim, Real>>& ts,
             const array_view<const complex_t, Dim + 1>& u_init)
      : grid_(grid), ts_(ts) {
    check(az_sim_create(ts->handle(), C, u_init.raw(), nullptr, &sim_), "Simulation");
  }
  ~Simulation() { az_sim_destroy(sim_); }
  Simulation(const Simulation&) = delete;
  Simulation& operator=(const Simulation&) = delete;
  void simulate_until(double t) { check(az_sim_simulate_until(sim_, t, nullptr), "Simulation::simulate_until"); }
  array_view<complex_t, Dim + 1> u() const {
    return array_view<complex_t, Dim + 1>(grid_.shape_fourier(Dim), static_cast<complex_t*>(az_sim_u(sim_)));
  }
  double time() const {
    double t = 0;
    check(az_sim_state(sim_, nullptr, &t, nullptr, nullptr), "Simulation::time");
    return t;
  }
  long long steps() const {
    long long n = 0;
    check(az_sim_state(sim_, nullptr, nullptr, &n, nullptr), "Simulation::steps");
    return n;
  }

 private:
  Grid<Dim> grid_;
  std::shared_ptr<SSP_RK3<Dim, Real>> ts_;
  az_sim sim_ = nullptr;
};

// FFT<Dim> (fft.hpp:37-121): unnormalised r2c forward / c2r backward over all
// axes, batched over n_vars = shape(0).
enum { FFT_FORWARD = AZ_FFT_FORWARD, FFT_BACKWARD = AZ_FFT_BACKWARD };
template <int Dim, typename Real = double>
class FFT {
 public:
  using complex_t = Complex<Real>;
  FFT(const array_view<complex_t, Dim + 1>& u_hat, const array_view<Real, Dim + 1>& u, int direction) {
    az_fft_desc d{};
    d.dim = Dim;
    d.n_vars = (long long)u.shape(0);
    for (int a = 0; a < Dim; ++a) d.shape[a] = (long long)u.shape(a + 1);
    d.transform_last = Dim;
    d.precision = sizeof(Real) == 8 ? AZ_PREC_F64 : AZ_PREC_F32;
    d.direction = direction;
    check(az_fft_create(&d, u_hat.raw(), u.raw(), &fft_), "FFT");
  }
  ~FFT() { az_fft_destroy(fft_); }
  FFT(const FFT&) = delete;
  FFT& operator=(const FFT&) = delete;
  void forward() { check(az_fft_forward(fft_, nullptr), "FFT::forward"); }
  void backward() { check(az_fft_backward(fft_, nullptr), "FFT::backward"); }
  std::size_t get_work_area_size() const { return az_fft_work_area_size(fft_); }
  void set_work_area(void* work) { check(az_fft_set_work_area(fft_, work), "FFT::set_work_area"); }

 private:
  az_fft fft_ = nullptr;
};

}  // namespace azb

#endif  // AZEBAN_B200_HPP_
