// A C++ driver over include/felbm_b200.hpp in the shape of the reference's
// felbm_gpu main loop (src/felbm_gpu_main.cu:586-594 forcing_factor_at,
// :735-748 the per-step body, :645-683 the asynchronous statistics harvest):
// read settings.cfg + params.cfg, log the fast-path switch mapping, upload an
// initial state, then per step set the forcing factor of step t, step, apply
// the mass correction, and launch / collect the flow statistics every
// log_skip steps. Test infrastructure: tests/test_*_drop_in.py builds it with
// g++ against the library and compares its final state with the CPU oracle.
//
//   drop_in_driver settings.cfg case_dir
//
// case_dir holds solid.bin (nx*ny*nz bytes, 1 = solid, x fastest) and
// h0.bin / g0.bin (19 n doubles, layout k*n + i); the driver writes h.bin,
// g.bin, series.txt (t, the six statistics) and switches.txt there.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "felbm_b200.hpp"

template <class T>
static std::vector<T> read_bin(const std::string& path) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) throw std::runtime_error("cannot open " + path);
  const std::streamsize bytes = in.tellg();
  in.seekg(0);
  std::vector<T> v((size_t)bytes / sizeof(T));
  in.read(reinterpret_cast<char*>(v.data()), bytes);
  return v;
}

template <class T>
static void write_bin(const std::string& path, const std::vector<T>& v) {
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::cerr << "usage: drop_in_driver settings.cfg case_dir\n";
    return 2;
  }
  const std::string dir = std::string(argv[2]) + "/";
  try {
    fe_params p;
    fe::check(fe_params_default(&p));
    fe_open_bnd ob{};
    fe_driver_cfg cfg;
    fe::read_cfg(argv[1], p, ob, cfg);
    {
      std::ofstream sw(dir + "switches.txt");
      sw << fe::switch_log(p);
    }
    const std::vector<uint8_t> solid = read_bin<uint8_t>(dir + "solid.bin");
    if ((int64_t)solid.size() != (int64_t)cfg.size_x * cfg.size_y * cfg.size_z)
      throw std::runtime_error("solid.bin does not match size_x * size_y * size_z");
    fe::MultiPhaseGPU gpu(p, cfg.size_x, cfg.size_y, cfg.size_z, solid.data(), cfg.gpu_device);
    const std::vector<double> h0 = read_bin<double>(dir + "h0.bin"), g0 = read_bin<double>(dir + "g0.bin");
    if ((int)h0.size() != gpu.state_size() || (int)g0.size() != gpu.state_size())
      throw std::runtime_error("initial state does not match the lattice");
    gpu.upload_state(h0.data(), g0.data());
    gpu.record_target_mass();
    // forcing_factor_at (felbm_gpu_main.cu:589-593)
    const double PI = 3.14159265358979323846;
    auto forcing_factor_at = [&](unsigned t) -> double {
      if (p.forcing_timedep == FE_FORCING_SINUSOIDAL) return std::sin(2.0 * PI * double(t) / p.forcing_period);
      if (p.forcing_timedep == FE_FORCING_SQUARE) {
        const double x = std::sin(2.0 * PI * double(t) / p.forcing_period);
        return (x < 0) ? -1.0 : ((x > 0) ? 1.0 : 0.0);
      }
      return 1.0;
    };
    const unsigned steps = (unsigned)cfg.max_iterations;
    const unsigned lskip = cfg.log_skip > 0 ? (unsigned)cfg.log_skip : 1u;
    std::ofstream series(dir + "series.txt");
    series << std::setprecision(17);
    long p_iter = -1;
    auto harvest = [&]() {
      if (!gpu.flow_stats_pending()) return;
      double s[6];
      gpu.flow_stats_collect(s);
      series << p_iter;
      for (double x : s) series << ' ' << x;
      series << '\n';
    };
    for (unsigned t = 0; t <= steps; ++t) {
      if (t % lskip == 0) harvest();
      if (t < steps) {
        gpu.set_forcing_factor(forcing_factor_at(t));
        gpu.step();
        gpu.apply_mass_correction();
        if ((t + 1) % lskip == 0) {
          harvest();
          gpu.flow_stats_launch();
          p_iter = (long)(t + 1);
        }
      }
    }
    harvest();
    std::vector<double> h, g;
    gpu.download_state(h, g);
    write_bin(dir + "h.bin", h);
    write_bin(dir + "g.bin", g);
    std::cout << "drop_in_driver: " << steps << " steps on " << gpu.size_sites() << " sites\n";
  } catch (const fe::Error& e) {
    std::cerr << "drop_in_driver: felbm_b200 error " << e.status << ": " << e.what() << "\n";
    return 10 + e.status;
  } catch (const std::exception& e) {
    std::cerr << "drop_in_driver: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
