// A C++ caller of the library through include/azeban_b200.hpp, written the
// way azeban's own code drives Equation<Dim>, TimeIntegrator<Dim> and
// Simulation<Dim> (include/azeban/equations/equation.hpp:27-56,
// include/azeban/evolution/ssp_rk3.hpp:48-64, src/azeban/simulation.cpp:89-102).
//
// usage: adapter_main <dim> <N> <f64|f32> <eps> <u_hat.bin> <out_prefix>
// Reads u_hat (complex128, the reference's layout), then writes
//   <out_prefix>_dudt.bin    dudt of u_hat (in place, as the reference allows)
//   <out_prefix>_dt.txt      Equation::dt(0.2) after that dudt
//   <out_prefix>_step.bin    u_hat after one SSP_RK3::integrate(0, 1, 0.2, u)
//   <out_prefix>_sim.bin     Simulation state after simulate_until(0.01)
//   <out_prefix>_sim.txt     its clock and step count
// all as complex128.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <memory>
#include <string>
#include <vector>

#include "azeban_b200.hpp"

namespace {

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    std::exit(2);
  }
}

std::vector<std::complex<double>> read_all(const std::string& path, std::size_t n) {
  std::vector<std::complex<double>> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(v[0])));
  if (!f) {
    std::fprintf(stderr, "cannot read %s\n", path.c_str());
    std::exit(2);
  }
  return v;
}

void write_all(const std::string& path, const std::vector<std::complex<double>>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(v[0])));
}

template <int Dim, typename Real>
int run(long long N, double eps, const std::string& in, const std::string& out) {
  using C = azb::Complex<Real>;
  const azb::Grid<Dim> grid(N);
  const auto shape = grid.shape_fourier(Dim);
  std::size_t n = 1;
  for (auto s : shape) n *= s;
  // SmoothCutoff1D as make_smooth_cutoff_1d builds it: eps / N, k0 = 2 pi sqrt(N)
  const azb::SmoothCutoff1D visc{eps / double(N), 1.0, 2 * 3.14159265358979323846 * std::sqrt(double(N))};
  auto equation = std::make_shared<azb::IncompressibleEuler<Dim, Real>>(grid, visc);

  const auto host = read_all(in, n);
  std::vector<C> h(n);
  for (std::size_t i = 0; i < n; ++i) h[i] = C{Real(host[i].real()), Real(host[i].imag())};
  C* d_u = nullptr;
  cuda_ok(cudaMalloc(&d_u, n * sizeof(C)), "cudaMalloc");
  auto reset = [&] { cuda_ok(cudaMemcpy(d_u, h.data(), n * sizeof(C), cudaMemcpyHostToDevice), "copy in"); };
  auto dump = [&](const C* dev, const std::string& path) {
    std::vector<C> r(n);
    cuda_ok(cudaMemcpy(r.data(), dev, n * sizeof(C), cudaMemcpyDeviceToHost), "copy out");
    std::vector<std::complex<double>> o(n);
    for (std::size_t i = 0; i < n; ++i) o[i] = {double(r[i].x), double(r[i].y)};
    write_all(path, o);
  };
  azb::array_view<C, Dim + 1> u(shape, d_u);
  azb::array_view<const C, Dim + 1> u_c(shape, d_u);

  // Equation<Dim>::dudt, in place, then dt(C)
  reset();
  equation->dudt(u, u_c, 0.0, 0.0, 0.2);
  dump(d_u, out + "_dudt.bin");
  std::ofstream(out + "_dt.txt") << std::scientific << std::setprecision(17) << equation->dt(0.2) << "\n";

  // TimeIntegrator<Dim>::integrate through the base class
  reset();
  std::shared_ptr<azb::TimeIntegrator<Dim, Real>> ts = std::make_shared<azb::SSP_RK3<Dim, Real>>(equation);
  const double dt = ts->integrate(0.0, 1.0, 0.2, u);
  dump(d_u, out + "_step.bin");
  std::ofstream(out + "_step.txt") << std::scientific << std::setprecision(17) << dt << "\n";

  // Simulation<Dim>::simulate_until
  reset();
  auto rk3 = std::make_shared<azb::SSP_RK3<Dim, Real>>(equation);
  azb::Simulation<Dim, Real> sim(grid, 0.2, rk3, u_c);
  sim.simulate_until(0.01);
  dump(sim.u().raw(), out + "_sim.bin");
  std::ofstream(out + "_sim.txt") << std::scientific << std::setprecision(17) << sim.time() << " "
                                  << sim.steps() << "\n";
  cudaFree(d_u);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s <dim> <N> <f64|f32> <eps> <u_hat.bin> <out_prefix>\n", argv[0]);
    return 1;
  }
  const int dim = std::atoi(argv[1]);
  const long long N = std::atoll(argv[2]);
  const std::string prec = argv[3];
  const double eps = std::atof(argv[4]);
  try {
    if (dim == 2) return prec == "f64" ? run<2, double>(N, eps, argv[5], argv[6]) : run<2, float>(N, eps, argv[5], argv[6]);
    if (dim == 3) return prec == "f64" ? run<3, double>(N, eps, argv[5], argv[6]) : run<3, float>(N, eps, argv[5], argv[6]);
  } catch (const azb::Error& e) {
    std::fprintf(stderr, "azb::Error %d: %s\n", int(e.status), e.what());
    return 3;
  }
  std::fprintf(stderr, "dim must be 2 or 3\n");
  return 1;
}
