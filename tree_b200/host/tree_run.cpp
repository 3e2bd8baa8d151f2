// tree_run.cpp -- host driver for the B200 force path with the reference's
// inputs and outputs: control.prm and input.xyz as Init reads them
// (main.f90:196-426), initial velocities as Vinit draws them
// (main.f90:709-790), the step loop with the TEMPORAL / RDF / Restart cadence
// (main.f90:123-160) on the device through tree_gpu_run, and the files
// ener###.dat (sample.f90:55-96), rdf###.dat (sample.f90:5-50) and
// res###.xyz (print.f90:67-106).  A res###.xyz is a valid input.xyz for a
// restarted run (rest != OFF), so states round-trip.
//
//   tree_run [--dir D] [--precision mixed|fp64] [--mac learned|fixed]
//            [--physics kelbg|ref] [--model FILE] [--eta E] [--seed S]
//            [--dry-run]
//
// --dry-run parses the inputs and prints them as JSON without touching the
// GPU.  The learned criterion reads a raw model file: TREE_GPU_MLP_PARAMS
// then TREE_GPU_MLP_STATS float32 values (tree_b200/data/mac_model.bin).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include <unistd.h>

#include "../../include/tree_gpu.h"

namespace {

constexpr double kTps = 1.0180505305371923e-1;  // ns per code time unit (data.f90:39)
constexpr double kKb = 8.617343e-5;              // eV/K (main.f90:393)
constexpr int kNref = 6;                         // vacuum thermostat reference (data.f90:38)

// Fortran list-directed input: each READ starts a new record and takes as
// many values as it needs, continuing onto following records.
struct ListReader {
  std::ifstream in;
  bool ok = true;
  explicit ListReader(const std::string& path) : in(path) { ok = (bool)in; }
  static std::vector<std::string> split(const std::string& line) {
    std::vector<std::string> t;
    std::string cur;
    for (char ch : line) {
      if (ch == ',' || ch == ' ' || ch == '\t' || ch == '\r') {
        if (!cur.empty()) t.push_back(cur);
        cur.clear();
      } else {
        cur += ch;
      }
    }
    if (!cur.empty()) t.push_back(cur);
    return t;
  }
  // values of one READ statement
  std::vector<std::string> read(size_t count) {
    std::vector<std::string> out;
    std::string line;
    while (out.size() < count && std::getline(in, line)) {
      std::vector<std::string> t = split(line);
      for (const std::string& s : t)
        if (out.size() < count) out.push_back(s);
    }
    if (out.size() < count) ok = false;
    return out;
  }
  void skip() { read(1); }
};

double num(const std::string& s) {
  std::string t = s;
  for (char& c : t)
    if (c == 'd' || c == 'D') c = 'e';  // Fortran double exponent
  return std::strtod(t.c_str(), nullptr);
}

struct Control {
  double q[2], xm[2];
  int64_t nt_el = 0, nt_ion = 0;
  double te = 0, ti = 0;
  double tmax = 0, trest = 0, tdump = 0, tsamp = 0, dt = 0;  // code units
  int kelbg = 0;
  double rs = 0;
  std::string rest;
  double dx_ee = 0, dx_ei = 0, dx_ii = 0;
  double sd_ratio = 0;
};

bool read_control(const std::string& path, Control& c) {
  ListReader r(path);
  if (!r.ok) return false;
  r.skip();
  r.skip();
  for (int i = 0; i < 2; ++i) c.q[i] = num(r.read(1)[0]);
  r.skip();
  for (int i = 0; i < 2; ++i) c.xm[i] = num(r.read(1)[0]);
  r.skip();
  c.nt_el = (int64_t)num(r.read(1)[0]);
  c.nt_ion = (int64_t)num(r.read(1)[0]);
  r.skip();
  c.te = num(r.read(1)[0]);
  c.ti = num(r.read(1)[0]);
  r.skip();
  std::vector<std::string> t = r.read(5);
  if (!r.ok) return false;
  c.tmax = num(t[0]) / kTps;
  c.trest = num(t[1]) / kTps;
  c.tdump = num(t[2]) / kTps;
  c.tsamp = num(t[3]) / kTps;
  c.dt = num(t[4]) / kTps;
  r.skip();
  t = r.read(2);
  if (!r.ok) return false;
  c.kelbg = (int)num(t[0]);
  c.rs = num(t[1]);
  r.skip();
  t = r.read(1);
  if (!r.ok) return false;
  c.rest = t[0];
  if (c.rest.size() >= 2 && (c.rest.front() == '\'' || c.rest.front() == '"'))
    c.rest = c.rest.substr(1, c.rest.size() - 2);
  r.skip();
  t = r.read(3);
  if (!r.ok) return false;
  c.dx_ee = num(t[0]);
  c.dx_ei = num(t[1]);
  c.dx_ii = num(t[2]);
  r.skip();
  t = r.read(1);
  if (!r.ok) return false;
  c.sd_ratio = num(t[0]);
  return r.ok;
}

struct Particles {
  std::vector<double> x, v;  // 3 per particle
  std::vector<int64_t> id;
};

// input.xyz: two header records, then NTel electron and NTion ion records
// "tag x y z id" (rest = OFF) or "tag x y z vx vy vz id" (a restart file).
bool read_xyz(const std::string& path, int64_t n, bool with_v, Particles& p) {
  ListReader r(path);
  if (!r.ok) return false;
  r.skip();
  r.skip();
  p.x.assign(3 * n, 0.0);
  p.v.assign(3 * n, 0.0);
  p.id.assign(n, 0);
  for (int64_t i = 0; i < n; ++i) {
    std::vector<std::string> t = r.read(with_v ? 8 : 5);
    if (!r.ok) return false;
    for (int k = 0; k < 3; ++k) p.x[3 * i + k] = num(t[1 + k]);
    if (with_v)
      for (int k = 0; k < 3; ++k) p.v[3 * i + k] = num(t[4 + k]);
    p.id[i] = (int64_t)num(t[with_v ? 7 : 4]);
  }
  return true;
}

// Vinit (main.f90:736-770): Gaussian components, rescaled per species so
// that sum m v^2 = kb (3N - Nref) T exactly.
void vinit(std::vector<double>& v, int64_t i0, int64_t n, double xm, double temp,
           std::mt19937_64& rng) {
  std::normal_distribution<double> nd(0.0, std::sqrt(temp > 0 ? temp : 1.0));
  double mv2 = 0.0;
  for (int64_t i = i0; i < i0 + n; ++i)
    for (int k = 0; k < 3; ++k) {
      double w = nd(rng);
      v[3 * i + k] = w;
      mv2 += xm * w * w;
    }
  if (n <= 0 || mv2 <= 0.0) return;
  const double t0 = mv2 / kKb / (double)(3 * n - kNref);
  const double lam = std::sqrt(temp / t0);
  for (int64_t i = i0; i < i0 + n; ++i)
    for (int k = 0; k < 3; ++k) v[3 * i + k] *= lam;
}

std::string es(double v) {  // Fortran ES14.6
  char b[32];
  std::snprintf(b, sizeof b, "%14.6E", v);
  return b;
}

void die(tree_gpu_handle* h, int rc, const char* what) {
  std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, h ? tree_gpu_last_error(h) : "");
  std::exit(1);
}

}  // namespace

int main(int argc, char** argv) {
  std::string dir = ".", model;
  int precision = TREE_GPU_PREC_MIXED, mac = TREE_GPU_MAC_LEARNED, physics = TREE_GPU_PHYS_KELBG;
  double eta = 3e-5;
  uint64_t seed = 1;
  bool dry = false;
  for (int a = 1; a < argc; ++a) {
    std::string s = argv[a];
    auto next = [&]() -> std::string { return a + 1 < argc ? argv[++a] : ""; };
    if (s == "--dir") dir = next();
    else if (s == "--precision") precision = next() == "fp64" ? TREE_GPU_PREC_FP64 : TREE_GPU_PREC_MIXED;
    else if (s == "--mac") mac = next() == "fixed" ? TREE_GPU_MAC_FIXED : TREE_GPU_MAC_LEARNED;
    else if (s == "--physics") physics = next() == "ref" ? TREE_GPU_PHYS_REF : TREE_GPU_PHYS_KELBG;
    else if (s == "--model") model = next();
    else if (s == "--eta") eta = std::atof(next().c_str());
    else if (s == "--seed") seed = std::strtoull(next().c_str(), nullptr, 10);
    else if (s == "--dry-run") dry = true;
    else {
      std::fprintf(stderr, "unknown argument %s\n", s.c_str());
      return 2;
    }
  }
  if (precision == TREE_GPU_PREC_FP64) mac = TREE_GPU_MAC_FIXED;
  if (model.empty()) {  // the model shipped next to the driver
    char exe[4096];
    const ssize_t len = readlink("/proc/self/exe", exe, sizeof exe - 1);
    std::string d = len > 0 ? std::string(exe, (size_t)len) : std::string(argv[0]);
    const size_t slash = d.rfind('/');
    d = slash == std::string::npos ? std::string(".") : d.substr(0, slash);
    model = d + "/data/mac_model.bin";
  }
  Control c;
  if (!read_control(dir + "/control.prm", c)) {
    std::fprintf(stderr, "cannot parse %s/control.prm\n", dir.c_str());
    return 1;
  }
  const int64_t n = c.nt_el + c.nt_ion;
  const bool restart = c.rest != "OFF";
  Particles p;
  if (!read_xyz(dir + "/input.xyz", n, restart, p)) {
    std::fprintf(stderr, "cannot parse %s/input.xyz\n", dir.c_str());
    return 1;
  }
  const double dt = c.dt;
  const int64_t ndump = std::llround(c.tdump / dt), nrest = std::llround(c.trest / dt),
                nsamp = std::llround(c.tsamp / dt);
  const int64_t nloop_max = std::llround((c.tmax + 0.5 * dt) / dt) - 1;
  if (dry) {
    std::printf("{\"nt_el\": %lld, \"nt_ion\": %lld, \"xm\": [%.17g, %.17g], \"te\": %.17g, "
                "\"ti\": %.17g, \"dt\": %.17g, \"ndump\": %lld, \"nrest\": %lld, "
                "\"nsamp\": %lld, \"nloop_max\": %lld, \"rs\": %.17g, \"rest\": \"%s\", "
                "\"dx\": [%.17g, %.17g, %.17g], \"sd_ratio\": %.17g, "
                "\"x_first\": [%.17g, %.17g, %.17g], \"id_last\": %lld}\n",
                (long long)c.nt_el, (long long)c.nt_ion, c.xm[0], c.xm[1], c.te, c.ti, dt,
                (long long)ndump, (long long)nrest, (long long)nsamp, (long long)nloop_max,
                c.rs, c.rest.c_str(), c.dx_ee, c.dx_ei, c.dx_ii, c.sd_ratio,
                n ? p.x[0] : 0.0, n ? p.x[1] : 0.0, n ? p.x[2] : 0.0,
                n ? (long long)p.id[n - 1] : 0LL);
    return 0;
  }
  if (ndump <= 0 || nrest <= 0 || nsamp <= 0 || nloop_max < 0) {
    std::fprintf(stderr, "tdump, trest, tsamp must be at least dt\n");
    return 1;
  }
  if (!restart) {
    std::mt19937_64 rng(seed);
    vinit(p.v, 0, c.nt_el, c.xm[0], c.te, rng);
    vinit(p.v, c.nt_el, c.nt_ion, c.xm[1], c.ti, rng);
  }
  tree_gpu_params prm{};
  prm.theta = c.sd_ratio;
  prm.rs = c.rs > 0 ? c.rs : 1.0;
  prm.te = c.te > 0 ? c.te : 1.0;
  prm.xm_el = c.xm[0];
  prm.xm_ion = c.xm[1];
  prm.dx_ei = c.dx_ei;
  prm.dx_ii = c.dx_ii;
  prm.physics = physics;
  prm.precision = precision;
  prm.mac = mac;
  tree_gpu_handle* h = nullptr;
  int rc = tree_gpu_create(&prm, c.nt_el, c.nt_ion, &h);
  if (rc) die(h, rc, "tree_gpu_create");
  if (mac == TREE_GPU_MAC_LEARNED) {
    std::vector<float> buf(TREE_GPU_MLP_PARAMS + TREE_GPU_MLP_STATS);
    std::FILE* f = std::fopen(model.c_str(), "rb");
    if (!f || std::fread(buf.data(), sizeof(float), buf.size(), f) != buf.size()) {
      std::fprintf(stderr, "cannot read model %s (use --model or --mac fixed)\n", model.c_str());
      return 1;
    }
    std::fclose(f);
    if ((rc = tree_gpu_mac_set_model(h, buf.data(), buf.data() + TREE_GPU_MLP_PARAMS)))
      die(h, rc, "tree_gpu_mac_set_model");
    if ((rc = tree_gpu_mac_config(h, (float)eta, 0.05f, 0.9f))) die(h, rc, "tree_gpu_mac_config");
  }
  const int64_t ne = c.nt_el;
  rc = tree_gpu_set_state(h, p.x.data(), p.v.data(), p.x.data() + 3 * ne, p.v.data() + 3 * ne);
  if (rc) die(h, rc, "tree_gpu_set_state");
  // TEMPORAL normalisation (main.f90:392-398)
  const double kbm_e = kKb * (double)(3 * c.nt_el - kNref), kbm_i = kKb * (double)(3 * c.nt_ion - kNref);
  const double kbm_e_rad = kKb * (double)(c.nt_el - kNref), kbm_e_cir = kKb * (double)(2 * c.nt_el - kNref);
  const double kbm_i_rad = kKb * (double)(c.nt_ion - kNref), kbm_i_cir = kKb * (double)(2 * c.nt_ion - kNref);
  std::FILE* ener = std::fopen((dir + "/ener000.dat").c_str(), "w");
  std::fprintf(ener, "# time(ns)-   T_el.  -  T_ion  -  T_el_radial  -  T_ion_radial -  "
                     "T_el_circumf  -  T_ion_circumf  -  Potential Energy  - Total energy  -  "
                     "Number of Rydberg atoms\n");
  std::vector<int64_t> rdf_ei(TREE_GPU_RDF_BINS, 0), rdf_ii(TREE_GPU_RDF_BINS, 0);
  std::vector<tree_gpu_sample> recs;
  std::vector<double> f(3 * n);
  int64_t nloop = 0;
  while (nloop <= nloop_max) {
    // run to the next RDF or Restart step, or to the end
    int64_t next = std::min((nloop / ndump + 1) * ndump, (nloop / nrest + 1) * nrest);
    next = std::min(next, nloop_max + 1);
    const int32_t steps = (int32_t)(next - nloop);
    recs.resize((size_t)(steps / nsamp + 2));
    int32_t nrec = 0;
    rc = tree_gpu_run(h, dt, steps, (int32_t)nsamp, recs.data(), (int32_t)recs.size(), &nrec,
                      rdf_ei.data(), rdf_ii.data());
    if (rc) die(h, rc, "tree_gpu_run");
    nloop = next;
    // TEMPORAL lines of the sample steps
    for (int32_t k = 0; k < nrec; ++k) {
      const tree_gpu_sample& s = recs[k];
      const double tnow = (double)s.nloop * dt;
      const double epot = s.epot_e + s.epot_i;
      std::fprintf(ener, "%s %s %s %s %s %s %s %s %s \n", es(tnow * kTps).c_str(),
                   es(s.mv2_el / kbm_e).c_str(), es(s.mv2_ion / kbm_i).c_str(),
                   es(s.rad_el / kbm_e_rad).c_str(), es(s.rad_ion / kbm_i_rad).c_str(),
                   es((s.mv2_el - s.rad_el) / kbm_e_cir).c_str(),
                   es((s.mv2_ion - s.rad_ion) / kbm_i_cir).c_str(), es(epot).c_str(),
                   es(0.5 * (s.mv2_el + s.mv2_ion) + epot).c_str());
    }
    if (nloop % ndump == 0) {  // RDF (sample.f90:5-50)
      char name[32];
      std::snprintf(name, sizeof name, "/rdf%03lld.dat", (long long)(nloop / ndump));
      std::FILE* r = std::fopen((dir + name).c_str(), "w");
      std::fprintf(r, "# R_ei,   RDF_ei       R_ii     RDF_ii     scaled RDF_ii\n");
      const double ntau = (double)ndump;
      for (int i = 0; i < TREE_GPU_RDF_BINS; ++i)
        std::fprintf(r, "%s %s %s %s \n", es(c.dx_ei * (i + 1)).c_str(),
                     es((double)rdf_ei[i] / ntau).c_str(), es(c.dx_ii * (i + 1)).c_str(),
                     es((double)rdf_ii[i] / ntau).c_str());
      std::fclose(r);
      std::fill(rdf_ei.begin(), rdf_ei.end(), 0);
      std::fill(rdf_ii.begin(), rdf_ii.end(), 0);
    }
    if (nloop % nrest == 0) {  // Restart (print.f90:67-106), then a new energy file
      if ((rc = tree_gpu_get_state(h, p.x.data(), p.v.data(), f.data(), p.x.data() + 3 * ne,
                                   p.v.data() + 3 * ne, f.data() + 3 * ne)))
        die(h, rc, "tree_gpu_get_state");
      const long long nfreq = (long long)(nloop / nrest);
      char name[32];
      std::snprintf(name, sizeof name, "/res%03lld.xyz", nfreq);
      std::FILE* r = std::fopen((dir + name).c_str(), "w");
      std::fprintf(r, " %lld\n frame = %lld   energy = 0\n", (long long)n, nfreq);
      for (int64_t i = 0; i < n; ++i) {
        std::fprintf(r, "%s  ", i < ne ? "P" : "O");
        for (int k = 0; k < 3; ++k) std::fprintf(r, "%s ", es(p.x[3 * i + k]).c_str());
        for (int k = 0; k < 3; ++k) std::fprintf(r, "%s ", es(p.v[3 * i + k]).c_str());
        std::fprintf(r, "%8lld\n", (long long)p.id[i]);
      }
      std::fclose(r);
      std::fclose(ener);
      std::snprintf(name, sizeof name, "/ener%03lld.dat", nfreq);
      ener = std::fopen((dir + name).c_str(), "w");
      std::fprintf(ener, "# time(ns)-   T_el.  -  T_ion  -  T_el_radial  -  T_ion_radial -  "
                         "T_el_circumf  -  T_ion_circumf  -  Potential Energy  - Total "
                         "energy  -  Number of Rydberg atoms\n");
    }
  }
  std::fclose(ener);
  tree_gpu_timing t{};
  tree_gpu_timings(h, &t);
  std::printf("steps %lld  build %.3f ms  walk %.3f ms  total %.3f ms  (%s)\n",
              (long long)nloop, t.ms_build, t.ms_walk, t.ms_total, tree_gpu_version());
  tree_gpu_destroy(h);
  return 0;
}
