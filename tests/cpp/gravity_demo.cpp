// A C++ host written against the Visitor API, driving the device path through
// include/paratreet_gpu.hpp (built and run by tests/test_cpp_facade.py).
//
//   gravity_demo copy  in.tipsy out.tipsy            read and write Tipsy (no GPU)
//   gravity_demo forces in.tipsy out.acc theta bucket [mixed]
//                                                    one force pass, .acc output
//   gravity_demo steps in.tipsy out.tipsy theta bucket dt n
//                                                    n Driver::run iterations
//   gravity_demo sph in.tipsy out.txt bucket         SPH density + pressure pass
//                                                    (u = 1 + i mod 7 / 10), one
//                                                    line per particle: density
//                                                    ax ay az pdv
//   gravity_demo sphsteps in.tipsy out.txt bucket dt n
//                                                    n SPH iterations (same u),
//                                                    one line per particle: x y z
//                                                    vx vy vz u u_pred
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "paratreet_gpu.hpp"

using namespace paratreet_gpu;

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s copy|forces|steps in out [theta bucket [dt n | mixed]]\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  try {
    TipsyHeader h;
    Particles p = read_tipsy(argv[2], &h);
    std::printf("read %d particles (gas %d, dark %d, star %d), time %.17g\n", h.nbodies, h.nsph, h.ndark,
                h.nstar, h.time);
    if (mode == "copy") {
      write_tipsy(argv[3], p, h.time);
      return 0;
    }
    Configuration conf;
    conf.theta = argc > 4 ? std::atof(argv[4]) : 0.7;
    conf.max_particles_per_leaf = argc > 5 ? std::atoi(argv[5]) : 16;
    if (mode == "forces") {
      if (argc > 6 && std::strcmp(argv[6], "mixed") == 0) conf.precision = PT_MIXED;
      Gravity g(conf);
      g.load(p);
      Accelerations a = run_gravity(g, GravityVisitor(Vector3D{0, 0, 0}, conf.theta));
      write_acc(argv[3], a);
      const pt_counters c = g.counters();
      std::printf("buckets %lld nodes %lld pp %llu pc %llu\n", (long long)c.n_buckets, (long long)c.n_nodes,
                  (unsigned long long)c.n_pp, (unsigned long long)c.n_pc);
      return 0;
    }
    if (mode == "steps" && argc > 7) {
      conf.max_timestep = std::atof(argv[6]);
      Gravity g(conf);
      g.load(p);
      g.run(std::atoi(argv[7]));
      g.state(p);
      write_tipsy(argv[3], p, h.time);
      return 0;
    }
    if (mode == "sph") {
      conf.max_particles_per_leaf = argc > 4 ? std::atoi(argv[4]) : 16;
      Gravity g(conf);
      g.load(p);
      std::vector<double> u(p.size());
      for (size_t i = 0; i < u.size(); i++) u[i] = 1.0 + (double)(i % 7) / 10.0;
      const Gravity::Sph s = g.sph_pressure(u);
      FILE* f = std::fopen(argv[3], "w");
      if (!f) throw Error(PT_E_ARG, "cannot open output");
      for (size_t i = 0; i < u.size(); i++)
        std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g\n", s.density[i], s.ax[i], s.ay[i], s.az[i], s.pdv[i]);
      std::fclose(f);
      return 0;
    }
    if (mode == "sphsteps" && argc > 6) {
      conf.max_particles_per_leaf = std::atoi(argv[4]);
      conf.max_timestep = std::atof(argv[5]);
      Gravity g(conf);
      g.load(p);
      Gravity::SphState s;
      s.u.resize(p.size());
      for (size_t i = 0; i < p.size(); i++) s.u[i] = 1.0 + (double)(i % 7) / 10.0;
      s.u_pred = s.u;  // src/Reader.C:90-91
      s.vpx = p.vx;
      s.vpy = p.vy;
      s.vpz = p.vz;
      g.sph_run(std::atoi(argv[6]), s);
      g.state(p);
      FILE* f = std::fopen(argv[3], "w");
      if (!f) throw Error(PT_E_ARG, "cannot open output");
      for (size_t i = 0; i < p.size(); i++)
        std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", p.x[i], p.y[i], p.z[i], p.vx[i],
                     p.vy[i], p.vz[i], s.u[i], s.u_pred[i]);
      std::fclose(f);
      return 0;
    }
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
  } catch (const Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
    return 1;
  }
}
