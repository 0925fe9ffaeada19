/* A C++ client of include/chainamps_b200_shim_core.hpp: one two-vertex
 * window read from MPX_matrix files, driven through the reference's seams --
 * the ARPACK MV callback on host std::complex<double> buffers, the lowest
 * eigenpair (HED), and the block SVD.
 *
 * usage: shim_window <dir> <nq> <chi> <max_trunc>
 *   <dir>/L.MPX_matrix, W.MPX_matrix, R.MPX_matrix, rules.i16, basis.i16,
 *   x.c128 (one vector in ARPACK order); writes y.c128 = H_eff x,
 *   allowed.i64, energy.f64, evec.c128, values.f64 (kept singular values). */
#include <complex>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "chainamps_b200_shim_core.hpp"

template <class T>
static std::vector<T> read_all(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    std::printf("cannot read %s\n", path.c_str());
    std::exit(2);
  }
  const std::streamsize n = f.tellg();
  f.seekg(0);
  std::vector<T> v((size_t)n / sizeof(T));
  f.read(reinterpret_cast<char*>(v.data()), n);
  return v;
}

template <class T>
static void write_all(const std::string& path, const T* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), (std::streamsize)(n * sizeof(T)));
}

int main(int argc, char** argv) {
  if (argc != 5) {
    std::printf("usage: %s <dir> <nq> <chi> <max_trunc>\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const int nq = std::stoi(argv[2]);
  const long chi = std::stol(argv[3]);
  const double trunc = std::stod(argv[4]);
  std::vector<int16_t> rules = read_all<int16_t>(dir + "/rules.i16");
  std::vector<int16_t> basis = read_all<int16_t>(dir + "/basis.i16");
  cmps_shim::Context ctx(0);
  cmps_shim::Tensor L = cmps_shim::load_tensor(dir + "/L.MPX_matrix", nq);
  cmps_shim::Tensor W = cmps_shim::load_tensor(dir + "/W.MPX_matrix", nq, basis);
  cmps_shim::Tensor R = cmps_shim::load_tensor(dir + "/R.MPX_matrix", nq);
  cmps_shim::TwoVertex window(ctx, rules, L, W, R);
  const size_t n = (size_t)window.size();
  std::vector<std::complex<double> > x = read_all<std::complex<double> >(dir + "/x.c128");
  if (x.size() != n) {
    std::printf("x has %zu values, the window %zu\n", x.size(), n);
    return 3;
  }
  // the reference's ARPACK loop hands the MV callback two workd slices
  std::vector<std::complex<double> > workd(2 * n);
  for (size_t i = 0; i < n; ++i) workd[i] = x[i];
  void (*mv)(const cmps_shim::TwoVertex*, std::complex<double>*, std::complex<double>*) = &cmps_shim::two_vertex_multiply;
  mv(&window, workd.data(), workd.data() + n);
  write_all(dir + "/y.c128", workd.data() + n, n);
  std::vector<int64_t> allowed = window.allowed_indices();
  write_all(dir + "/allowed.i64", allowed.data(), allowed.size());
  std::vector<std::complex<double> > evec(n);
  int matvecs = 0;
  const double e = window.lowest(nullptr, evec.data(), 1e-12, &matvecs, 50, 32);
  write_all(dir + "/energy.f64", &e, 1);
  write_all(dir + "/evec.c128", evec.data(), n);
  cmps_shim::SvdFactors f = window.svd(chi, trunc);
  write_all(dir + "/values.f64", f.values.data(), f.values.size());
  std::printf("window n=%zu energy=%.15g matvecs=%d kept=%ld\n", n, e, matvecs, (long)f.kept);
  return 0;
}
