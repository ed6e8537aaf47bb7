// paratreet_gpu.hpp -- C++ host facade over the C ABI of pt_gravity.h, for host
// code written against ParaTreeT's Visitor / Data API.  Header-only, C++17;
// link with libpt_gravity.so.
//
//   paratreet_gpu::GravityVisitor   examples/GravityVisitor.h:9-231 -- the same
//                                   static traits and (offset, theta) constructor
//   paratreet_gpu::Configuration    the fields of src/Configuration.h:100-150
//                                   this path reads (bucket size, theta, dt,
//                                   periodic box)
//   paratreet_gpu::Gravity          one simulation: load (Reader::load),
//                                   startDown<GravityVisitor> (src/Partition.h:
//                                   129-134), run (Driver::run, src/Driver.h:
//                                   183-251), accelerations
//                                   (outputParticleAccelerations)
//   paratreet_gpu::run_gravity      ExMain::traversalFn (examples/Gravity.C:29-52)
//   read_tipsy / write_tipsy /      src/Reader.C:11-116, src/Writer.C:31-159
//   write_acc
//
// Errors from the library become paratreet_gpu::Error (code = PT_E_*).
#ifndef PARATREET_GPU_HPP_
#define PARATREET_GPU_HPP_

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "pt_gravity.h"

namespace paratreet_gpu {

struct Vector3D {
  double x = 0.0, y = 0.0, z = 0.0;
};

class Error : public std::runtime_error {
 public:
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// GravityVisitor of examples/GravityVisitor.h: traits, offset and theta.  The
// open / node / leaf bodies run on the device; the traits are those the
// reference's traversers read.
struct GravityVisitor {
  static constexpr bool CallSelfLeaf = true;
  static constexpr bool ForceEvenDepth = true;
  static constexpr bool TargetMustBeLeaf = true;
  static constexpr double opening_geometry_factor_squared = 4.0 / 3.0;
  Vector3D offset;
  double theta = 0.7;
  GravityVisitor() = default;
  GravityVisitor(Vector3D offseti, double thetai) : offset(offseti), theta(thetai) {}
  double gravity_factor() const { return opening_geometry_factor_squared / (theta * theta); }
};

// Particle SoA in the caller's order (Particle::order).  type: 0 gas, 1 dark,
// 2 star (only the Tipsy functions read it).
struct Particles {
  std::vector<double> x, y, z, vx, vy, vz, mass, soft;
  std::vector<int8_t> type;
  size_t size() const { return x.size(); }
  void resize(size_t n) {
    for (auto* v : {&x, &y, &z, &vx, &vy, &vz, &mass, &soft}) v->assign(n, 0.0);
    type.assign(n, 1);
  }
};

struct Accelerations {
  std::vector<double> ax, ay, az;
  std::vector<double> pot;       // the reference's potential (node() terms)
  std::vector<double> pot_full;  // every interaction's potential
};

struct Configuration {
  int max_particles_per_leaf = 16;  // -l
  double theta = 0.7;
  double max_timestep = 1e-5;       // -j
  int precision = PT_FP64;          // PT_FP64 (reference-exact), PT_MIXED or PT_FP64_LISTS
  int integrator = PT_KKD;          // PT_KKD (Driver::run) or PT_KDK
  int device = 0;
  bool periodic = false;            // bPeriodic
  double fPeriod = 1.0;             // dxPeriod (cubic box)
  int nReplicas = 0;
  double fEwCut = 2.6;              // examples/Ewald.h:26
  double dEwhCut = 2.8;             // examples/Ewald.C:86
};

class Gravity {
 public:
  explicit Gravity(const Configuration& c) : conf_(c) {
    pt_config cfg;
    check(pt_config_default(&cfg), "pt_config_default");
    cfg.theta = c.theta;
    cfg.bucket = c.max_particles_per_leaf;
    cfg.dt_max = c.max_timestep;
    cfg.precision = c.precision;
    cfg.integrator = c.integrator;
    cfg.device = c.device;
    cfg.periodic = c.periodic ? 1 : 0;
    cfg.period = c.fPeriod;
    cfg.n_replicas = c.nReplicas;
    cfg.ewald_rcut = c.fEwCut;
    cfg.ewald_hcut = c.dEwhCut;
    int rc = pt_create(&cfg, &h_);
    if (rc != PT_OK) throw Error(rc, "pt_create failed (no CUDA device or invalid configuration)");
  }
  ~Gravity() {
    if (h_) pt_destroy(h_);
  }
  Gravity(const Gravity&) = delete;
  Gravity& operator=(const Gravity&) = delete;
  Gravity(Gravity&& o) noexcept : conf_(o.conf_), h_(std::exchange(o.h_, nullptr)), n_(o.n_) {}

  pt_handle* handle() const { return h_; }
  size_t size() const { return n_; }

  // Reader::load: particles to the device.
  void load(const Particles& p) {
    n_ = p.size();
    check(pt_set_particles(h_, (int64_t)n_, p.x.data(), p.y.data(), p.z.data(), p.vx.data(), p.vy.data(),
                           p.vz.data(), p.mass.data(), p.soft.data()),
          "pt_set_particles");
  }

  // Partition::startDown<GravityVisitor>: one force pass (tree build included).
  // Replica offsets come from the periodic configuration, as traversalFn makes
  // them; a visitor with a non-zero offset is rejected.
  void startDown(const GravityVisitor& v) { startDown(v, -1, -1); }
  void startDown(const GravityVisitor& v, int64_t b0, int64_t b1) {
    if (v.offset.x != 0.0 || v.offset.y != 0.0 || v.offset.z != 0.0)
      throw Error(PT_E_ARG, "replica offsets are generated by the periodic configuration");
    if (v.theta != conf_.theta) {
      check(pt_set_theta(h_, v.theta), "pt_set_theta");
      conf_.theta = v.theta;
    }
    if (b0 < 0) check(pt_compute_forces(h_), "pt_compute_forces");
    else check(pt_compute_forces_range(h_, b0, b1), "pt_compute_forces_range");
  }

  Accelerations accelerations() const {
    Accelerations a;
    for (auto* v : {&a.ax, &a.ay, &a.az, &a.pot, &a.pot_full}) v->assign(n_, 0.0);
    check(pt_get_accel(h_, a.ax.data(), a.ay.data(), a.az.data(), a.pot.data(), a.pot_full.data()),
          "pt_get_accel");
    return a;
  }

  // Driver::run: iterations of forces, kick, perturb.
  void run(int iterations) { check(pt_step(h_, iterations), "pt_step"); }

  // Positions and velocities into p (masses, softening and types kept).
  void state(Particles& p) const {
    if (p.size() != n_) p.resize(n_);
    check(pt_get_state(h_, p.x.data(), p.y.data(), p.z.data(), p.vx.data(), p.vy.data(), p.vz.data()),
          "pt_get_state");
  }

  // The SPH example's traversalFn (examples/SPH.C:74-101) on these
  // particles: startUpAndDown<DensityVisitor> + DensityFn (density, ball^2),
  // and with internal energies u also startDown<PressureVisitor> + ForceFn +
  // the opposing effects (pressure accelerations, PdV work).
  struct Sph {
    std::vector<double> density, ball_sq, ax, ay, az, pdv;
  };
  Sph sph_density() {
    Sph s;
    s.density.assign(n_, 0.0);
    s.ball_sq.assign(n_, 0.0);
    check(pt_sph_density(h_, s.density.data(), s.ball_sq.data(), nullptr, nullptr), "pt_sph_density");
    return s;
  }
  Sph sph_pressure(const std::vector<double>& u) {
    if (u.size() != n_) throw Error(PT_E_ARG, "one internal energy per particle");
    Sph s;
    for (auto* v : {&s.density, &s.ax, &s.ay, &s.az, &s.pdv}) v->assign(n_, 0.0);
    check(pt_sph_pressure(h_, u.data(), s.density.data(), s.ax.data(), s.ay.data(), s.az.data(), s.pdv.data()),
          "pt_sph_pressure");
    return s;
  }

  // The SPH example's Driver::run: iterations of the density pass, the
  // pressure pass and Particle::kick / perturb with the internal-energy
  // updates (dt = max_timestep).  The SPH fields of every particle in caller
  // order; start u_pred = u and v_pred = the velocities (src/Reader.C:90-91).
  struct SphState {
    std::vector<double> u, u_pred, vpx, vpy, vpz;
  };
  void sph_run(int iterations, SphState& s) {
    for (auto* v : {&s.u, &s.u_pred, &s.vpx, &s.vpy, &s.vpz})
      if (v->size() != n_) throw Error(PT_E_ARG, "one SPH state value per particle");
    check(pt_sph_step(h_, iterations, s.u.data(), s.u_pred.data(), s.vpx.data(), s.vpy.data(), s.vpz.data()),
          "pt_sph_step");
  }

  pt_counters counters() const {
    pt_counters c;
    check(pt_get_counters(h_, &c), "pt_get_counters");
    return c;
  }

 private:
  void check(int rc, const char* what) const {
    if (rc != PT_OK) throw Error(rc, std::string(what) + ": " + (h_ ? pt_last_error(h_) : ""));
  }
  Configuration conf_;
  pt_handle* h_ = nullptr;
  size_t n_ = 0;
};

// ExMain::traversalFn for this path: one startDown<GravityVisitor> over every
// bucket (with the replica walks and the Ewald correction when periodic), then
// the accelerations that outputParticleAccelerations would write.
inline Accelerations run_gravity(Gravity& g, const GravityVisitor& v) {
  g.startDown(v);
  return g.accelerations();
}

// ------------------------------------------------------------------ Tipsy I/O
struct TipsyHeader {
  double time = 0.0;
  int nbodies = 0, ndim = 3, nsph = 0, ndark = 0, nstar = 0;
};

namespace detail {
inline bool host_little_endian() {
  const uint16_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}
// value of the n-byte field at p, stored big-endian (swap) or in host order
template <typename T>
T get(const unsigned char* p, bool swap) {
  unsigned char b[sizeof(T)];
  for (size_t i = 0; i < sizeof(T); i++) b[i] = swap ? p[sizeof(T) - 1 - i] : p[i];
  T v;
  std::memcpy(&v, b, sizeof(T));
  return v;
}
template <typename T>
void put_be(std::vector<unsigned char>& out, T v) {
  unsigned char b[sizeof(T)];
  std::memcpy(b, &v, sizeof(T));
  const bool le = host_little_endian();
  for (size_t i = 0; i < sizeof(T); i++) out.push_back(le ? b[sizeof(T) - 1 - i] : b[i]);
}
// record sizes: mass + 3 pos + 3 vel + tail floats (gas 5, dark 2, star 4)
inline size_t rec_bytes(int kind, size_t pos, size_t vel) {
  static const int tail[3] = {5, 2, 4};
  return 4 + 3 * pos + 3 * vel + 4 * (size_t)tail[kind];
}
}  // namespace detail

// Reader::load (src/Reader.C:11-107): standard (big-endian) or native byte
// order, float or double positions / velocities (detected from the file size);
// softening from gas hsmooth and dark eps, zero for stars; dSoft >= 0 replaces
// every softening (Reader::setSoft).
inline Particles read_tipsy(const std::string& path, TipsyHeader* hdr = nullptr, double dSoft = -1.0) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw Error(PT_E_ARG, "cannot open " + path);
  std::vector<unsigned char> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  if (buf.size() < 32) throw Error(PT_E_ARG, path + ": not a Tipsy file (short header)");
  TipsyHeader h;
  bool swap = false, ok = false;
  for (int attempt = 0; attempt < 2 && !ok; attempt++) {
    swap = (attempt == 0) == detail::host_little_endian();  // big-endian first
    h.time = detail::get<double>(&buf[0], swap);
    h.nbodies = detail::get<int32_t>(&buf[8], swap);
    h.ndim = detail::get<int32_t>(&buf[12], swap);
    h.nsph = detail::get<int32_t>(&buf[16], swap);
    h.ndark = detail::get<int32_t>(&buf[20], swap);
    h.nstar = detail::get<int32_t>(&buf[24], swap);
    ok = h.nbodies >= 0 && h.nsph >= 0 && h.ndark >= 0 && h.nstar >= 0 &&
         h.nbodies == h.nsph + h.ndark + h.nstar && h.ndim >= 1 && h.ndim <= 3;
  }
  if (!ok) throw Error(PT_E_ARG, path + ": not a Tipsy file (inconsistent header)");
  const int cnt[3] = {h.nsph, h.ndark, h.nstar};
  size_t pw = 0, vw = 0;
  const size_t widths[3][2] = {{4, 4}, {8, 4}, {8, 8}};
  for (auto& wv : widths) {
    size_t tot = 32;
    for (int k = 0; k < 3; k++) tot += (size_t)cnt[k] * detail::rec_bytes(k, wv[0], wv[1]);
    if (tot == buf.size()) {
      pw = wv[0];
      vw = wv[1];
      break;
    }
  }
  if (!pw) throw Error(PT_E_ARG, path + ": file size matches no Tipsy layout");
  Particles p;
  p.resize((size_t)h.nbodies);
  size_t off = 32, i = 0;
  auto real = [&](size_t w) {
    double v = (w == 8) ? detail::get<double>(&buf[off], swap) : (double)detail::get<float>(&buf[off], swap);
    off += w;
    return v;
  };
  for (int k = 0; k < 3; k++) {
    for (int j = 0; j < cnt[k]; j++, i++) {
      p.mass[i] = real(4);
      p.x[i] = real(pw);
      p.y[i] = real(pw);
      p.z[i] = real(pw);
      p.vx[i] = real(vw);
      p.vy[i] = real(vw);
      p.vz[i] = real(vw);
      double t[5] = {0, 0, 0, 0, 0};
      const int nt = (k == 0) ? 5 : (k == 1) ? 2 : 4;
      for (int q = 0; q < nt; q++) t[q] = real(4);
      p.soft[i] = (k == 0) ? t[2] : (k == 1) ? t[0] : 0.0;  // hsmooth / eps / unset
      p.type[i] = (int8_t)k;
    }
  }
  if (dSoft >= 0.0)
    for (auto& s : p.soft) s = dSoft;
  if (hdr) *hdr = h;
  return p;
}

// TipsyWriter::do_write (src/Writer.C:87-159): standard Tipsy, double
// positions and velocities, gas / dark / star in particle order by type;
// only mass, position and velocity are filled.
inline void write_tipsy(const std::string& path, const Particles& p, double time) {
  std::vector<unsigned char> out;
  int cnt[3] = {0, 0, 0};
  for (size_t i = 0; i < p.size(); i++) cnt[p.type.empty() ? 1 : p.type[i]]++;
  detail::put_be<double>(out, time);
  detail::put_be<int32_t>(out, (int32_t)p.size());
  detail::put_be<int32_t>(out, 3);
  for (int k = 0; k < 3; k++) detail::put_be<int32_t>(out, cnt[k]);
  detail::put_be<int32_t>(out, 0);
  for (int k = 0; k < 3; k++) {
    const int nt = (k == 0) ? 5 : (k == 1) ? 2 : 4;
    for (size_t i = 0; i < p.size(); i++) {
      if ((p.type.empty() ? 1 : p.type[i]) != k) continue;
      detail::put_be<float>(out, (float)p.mass[i]);
      for (double v : {p.x[i], p.y[i], p.z[i], p.vx[i], p.vy[i], p.vz[i]}) detail::put_be<double>(out, v);
      for (int q = 0; q < nt; q++) detail::put_be<float>(out, 0.0f);
    }
  }
  std::ofstream f(path, std::ios::binary);
  if (!f) throw Error(PT_E_ARG, "cannot write " + path);
  f.write(reinterpret_cast<const char*>(out.data()), (std::streamsize)out.size());
}

// Writer::do_write (src/Writer.C:31-72): N, then the x, y, z blocks, %.14g.
inline void write_acc(const std::string& path, const Accelerations& a) {
  FILE* fp = std::fopen(path.c_str(), "w");
  if (!fp) throw Error(PT_E_ARG, "cannot write " + path);
  std::fprintf(fp, "%d\n", (int)a.ax.size());
  for (const auto* v : {&a.ax, &a.ay, &a.az})
    for (double x : *v) std::fprintf(fp, "%.14g\n", x);
  std::fclose(fp);
}

}  // namespace paratreet_gpu

#endif  // PARATREET_GPU_HPP_
