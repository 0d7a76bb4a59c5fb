// heom_scan: a whole 2DES delay scan in one process, replacing the reference's
// three-stage workflow
//   script/IO-scripts/gen_2d_data.sh:1-64    writes 2d-input/key_{tau}_{T}.key from
//                                            key.key-tmpl (TAU1..3, T_END substituted),
//   script/cpu-script/submit_jobs.sh:49-67   runs one CPU_2DES process per key file,
//                                            stdout -> 2d-output/out_{tau}_{T}.out,
// with batched GPU propagation.
//
//   heom_scan --input-dir DIR --output-dir DIR [options]
//   heom_scan --template key.key-tmpl --key-dir DIR --output-dir DIR
//             [--t0 210] [--propagate 600] [--tau-step 10] [--tau-bound 600] [--T 0,100]
//             [options]
//   options: --precision fp32-bulk|fp64|fp64-exact (default fp32-bulk)
//            --device D   --full-precision   --dry-run
//
// Directory mode reads every *.key file of DIR, groups the files that differ only in
// pulse central times and end time (heom_problem_scan_compatible: same system, same
// disorder seed, hence the same samples), and runs each group as one heom_run_scan
// batch per disorder sample, averaging over samples as CPU_2DES.cpp:50-89 does.  Each
// key_X.key gives out_X.out (other names: <stem>.out) with CPU_2DES's lines
// ("%.6e %.6e" in iostream scientific form; --full-precision prints 17 digits).
// fp64-exact runs every key on the bit-exact path (byte-identical files to the reference
// build); fp32-bulk and fp64 agree with it to the documented tolerances.
//
// Template mode first writes the key files exactly as gen_2d_data.sh does (same names,
// same substitutions: rephasing tau2 = t0 + i for i = 0..bound, non-rephasing
// tau1 = t0 + |i| for i = -bound..-step, tau3 = t0 + |i| + T, t_end = tau3 + propagate)
// and then runs directory mode on them.
//
// --dry-run parses and groups the keys and prints the plan without touching a GPU.
// Exit status: 0 when every key produced its output, 1 otherwise (errors on stderr).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "heom.h"

namespace fs = std::filesystem;

namespace {

struct Key {
  std::string path, out_name;
  heom_problem *prob = nullptr;
  heom_problem_info info{};
};

struct Opts {
  std::string in_dir, out_dir, tmpl, key_dir;
  double t0 = 210, propagate = 600, tau_step = 10, tau_bound = 600;
  std::vector<std::string> T = {"0"};
  int precision = HEOM_FP32_BULK, device = 0, digits = 6;
  bool dry = false;
};

int usage(const char *argv0) {
  std::fprintf(stderr,
               "usage: %s --input-dir DIR --output-dir DIR [--precision fp32-bulk|fp64|fp64-exact] [--device D]\n"
               "          [--full-precision] [--dry-run]\n"
               "       %s --template key.key-tmpl --key-dir DIR --output-dir DIR [--t0 210] [--propagate 600]\n"
               "          [--tau-step 10] [--tau-bound 600] [--T 0,100,...] [options]\n",
               argv0, argv0);
  return 2;
}

// Numbers as bc prints the sums of gen_2d_data.sh: integers without a decimal point,
// otherwise the shortest form that reads back to the same double.
std::string num(double v) {
  char b[64];
  if (v == (double)(long long)v && std::fabs(v) < 1e15) {
    std::snprintf(b, sizeof b, "%lld", (long long)v);
    return b;
  }
  for (int prec = 1; prec <= 17; prec++) {
    std::snprintf(b, sizeof b, "%.*f", prec, v);
    if (std::strtod(b, nullptr) == v) break;
  }
  return b;
}

std::string out_name_for(const std::string &key_path) {
  std::string stem = fs::path(key_path).stem().string();
  if (stem.rfind("key", 0) == 0) stem = "out" + stem.substr(3);
  return stem + ".out";
}

void replace_all(std::string &s, const std::string &from, const std::string &to) {
  for (size_t p = s.find(from); p != std::string::npos; p = s.find(from, p + to.size())) s.replace(p, from.size(), to);
}

// gen_2d_data.sh:37-61: write the key files of a delay scan from the template.
bool write_template_keys(const Opts &o) {
  std::ifstream f(o.tmpl);
  if (!f) {
    std::fprintf(stderr, "heom_scan: cannot read template %s\n", o.tmpl.c_str());
    return false;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  std::error_code ec;
  fs::create_directories(o.key_dir, ec);
  auto emit = [&](double tau1, double tau2, double tau3, double t_end, const std::string &name) {
    std::string k = text;
    replace_all(k, "TAU1", num(tau1));
    replace_all(k, "TAU2", num(tau2));
    replace_all(k, "TAU3", num(tau3));
    replace_all(k, "T_END", num(t_end));
    std::ofstream out(fs::path(o.key_dir) / name);
    out << k;
    return (bool)out;
  };
  bool ok = true;
  for (const std::string &ts : o.T) {
    const double t = std::strtod(ts.c_str(), nullptr);
    for (double i = 0; i <= o.tau_bound; i += o.tau_step) // rephasing: pulse 1 first
      ok &= emit(o.t0, o.t0 + i, o.t0 + i + t, o.t0 + i + t + o.propagate, "key_" + num(i) + "_" + ts + ".key");
    for (double i = -o.tau_bound; i < 0; i += o.tau_step) { // non-rephasing: pulse 2 first
      const double a = -i;
      ok &= emit(o.t0 + a, o.t0, o.t0 + a + t, o.t0 + a + t + o.propagate, "key_" + num(i) + "_" + ts + ".key");
    }
  }
  if (!ok) std::fprintf(stderr, "heom_scan: writing key files to %s failed\n", o.key_dir.c_str());
  return ok;
}

bool write_out(const Opts &o, const Key &k, const double *P, int n) {
  std::ofstream out(fs::path(o.out_dir) / k.out_name);
  out << std::scientific << std::setprecision(o.digits);
  for (int j = 0; j < n; j++) out << P[2 * j] << " " << P[2 * j + 1] << '\n'; // CPU_2DES.cpp:91
  if (!out) std::fprintf(stderr, "heom_scan: writing %s failed\n", k.out_name.c_str());
  return (bool)out;
}

// One key on the bit-exact path, samples averaged as CPU_2DES.cpp:50-89.
bool run_exact(const Opts &o, Key &k) {
  heom_problem_reset_rng(k.prob);
  int rc = heom_problem_prepare_sample(k.prob);
  heom_opts opts{};
  opts.precision = HEOM_FP64_EXACT;
  opts.device = o.device;
  opts.max_points = 1;
  heom_plan *plan = nullptr;
  if (!rc) rc = heom_plan_create(k.prob, &opts, &plan);
  const int cap = std::max(k.info.n_record, 1);
  std::vector<double> P(2 * (size_t)cap, 0.0), p(2 * (size_t)cap, 0.0);
  int n = 0;
  for (int s = 0; !rc && s < k.info.n_sample; s++) {
    if (s > 0) {
      rc = heom_problem_prepare_sample(k.prob);
      if (!rc) rc = heom_plan_update(plan, k.prob);
    }
    if (!rc) rc = heom_run_2des(plan, p.data(), nullptr, cap, &n);
    for (int j = 0; !rc && j < 2 * n; j++) P[j] += p[j] / k.info.n_sample;
  }
  if (plan) heom_plan_destroy(plan);
  if (rc) {
    std::fprintf(stderr, "heom_scan: %s: %s\n", k.path.c_str(), heom_last_error());
    return false;
  }
  return write_out(o, k, P.data(), n);
}

// A group of scan-compatible keys as one batch per sample.
bool run_group(const Opts &o, std::vector<Key *> &g) {
  heom_problem *rep = g[0]->prob;
  const int n = (int)g.size();
  std::vector<heom_scan_point> pts(n);
  for (int i = 0; i < n; i++) {
    const heom_problem_info &f = g[i]->info;
    pts[i] = heom_scan_point{f.tau[0], f.tau[1], f.tau[2], f.t_end, 0};
  }
  heom_problem_reset_rng(rep);
  int rc = heom_problem_prepare_sample(rep); // the first draws precede the plan, as in CPU_2DES
  heom_opts opts{};
  opts.precision = o.precision;
  opts.device = o.device;
  opts.max_points = n;
  heom_plan *plan = nullptr;
  if (!rc) rc = heom_plan_create(rep, &opts, &plan);
  std::vector<long long> off(n);
  std::vector<int> cnt(n);
  long long total = 0;
  if (!rc) rc = heom_scan_layout(plan, pts.data(), n, off.data(), cnt.data(), &total);
  std::vector<double> P, p;
  if (!rc) {
    P.assign(2 * (size_t)std::max(total, 1LL), 0.0);
    p.assign(P.size(), 0.0);
  }
  const int ns = g[0]->info.n_sample;
  for (int s = 0; !rc && s < ns; s++) {
    if (s > 0) {
      rc = heom_problem_prepare_sample(rep);
      if (!rc) rc = heom_plan_update(plan, rep);
    }
    if (!rc) rc = heom_run_scan(plan, pts.data(), n, p.data(), off.data(), cnt.data());
    for (size_t j = 0; !rc && j < 2 * (size_t)total; j++) P[j] += p[j] / ns;
  }
  if (plan) heom_plan_destroy(plan);
  if (rc) {
    std::fprintf(stderr, "heom_scan: group of %s: %s\n", g[0]->path.c_str(), heom_last_error());
    return false;
  }
  bool ok = true;
  for (int i = 0; i < n; i++) ok &= write_out(o, *g[i], P.data() + 2 * off[i], cnt[i]);
  return ok;
}

} // namespace

int main(int argc, char **argv) {
  Opts o;
  for (int a = 1; a < argc; a++) {
    const std::string s = argv[a];
    auto val = [&](void) -> const char * { return a + 1 < argc ? argv[++a] : nullptr; };
    const char *v = nullptr;
    if (s == "--full-precision") o.digits = 17;
    else if (s == "--dry-run") o.dry = true;
    else if (!(v = val())) return usage(argv[0]);
    else if (s == "--input-dir") o.in_dir = v;
    else if (s == "--output-dir") o.out_dir = v;
    else if (s == "--template") o.tmpl = v;
    else if (s == "--key-dir") o.key_dir = v;
    else if (s == "--t0") o.t0 = std::strtod(v, nullptr);
    else if (s == "--propagate") o.propagate = std::strtod(v, nullptr);
    else if (s == "--tau-step") o.tau_step = std::strtod(v, nullptr);
    else if (s == "--tau-bound") o.tau_bound = std::strtod(v, nullptr);
    else if (s == "--device") o.device = std::atoi(v);
    else if (s == "--T") {
      o.T.clear();
      std::stringstream ts(v);
      for (std::string t; std::getline(ts, t, ',');)
        if (!t.empty()) o.T.push_back(t);
    } else if (s == "--precision") {
      const std::string p = v;
      if (p == "fp64-exact") o.precision = HEOM_FP64_EXACT;
      else if (p == "fp64") o.precision = HEOM_FP64;
      else if (p == "fp32-bulk") o.precision = HEOM_FP32_BULK;
      else return usage(argv[0]);
    } else {
      std::fprintf(stderr, "heom_scan: unknown option '%s'\n", s.c_str());
      return usage(argv[0]);
    }
  }
  if (!o.tmpl.empty()) {
    if (o.key_dir.empty() || o.tau_step <= 0) return usage(argv[0]);
    if (!write_template_keys(o)) return 1;
    o.in_dir = o.key_dir;
  }
  if (o.in_dir.empty() || o.out_dir.empty()) return usage(argv[0]);

  std::vector<std::string> paths;
  std::error_code ec;
  for (const auto &e : fs::directory_iterator(o.in_dir, ec))
    if (e.is_regular_file() && e.path().extension() == ".key") paths.push_back(e.path().string());
  if (ec) {
    std::fprintf(stderr, "heom_scan: cannot list %s: %s\n", o.in_dir.c_str(), ec.message().c_str());
    return 1;
  }
  std::sort(paths.begin(), paths.end());
  bool ok = true;
  std::vector<Key> keys;
  keys.reserve(paths.size());
  for (const std::string &path : paths) {
    Key k;
    k.path = path;
    k.out_name = out_name_for(path);
    if (int rc = heom_problem_from_key(path.c_str(), 0, &k.prob)) {
      std::fprintf(stderr, "heom_scan: %s: %s (%d)\n", path.c_str(), heom_last_error(), rc);
      ok = false;
      continue;
    }
    heom_problem_info_get(k.prob, &k.info);
    keys.push_back(k);
  }
  std::vector<std::vector<Key *>> groups;
  for (Key &k : keys) {
    bool placed = false;
    for (auto &g : groups)
      if (heom_problem_scan_compatible(g[0]->prob, k.prob) == 1) {
        g.push_back(&k);
        placed = true;
        break;
      }
    if (!placed) groups.push_back({&k});
  }
  if (o.dry) {
    std::printf("%zu key files, %zu scan groups\n", keys.size(), groups.size());
    for (size_t i = 0; i < groups.size(); i++) {
      std::printf("group %zu: %zu points, %d samples\n", i, groups[i].size(), groups[i][0]->info.n_sample);
      for (const Key *k : groups[i])
        std::printf("  %s -> %s  tau %s %s %s  t_end %s  records %d\n", fs::path(k->path).filename().c_str(),
                    k->out_name.c_str(), num(k->info.tau[0]).c_str(), num(k->info.tau[1]).c_str(),
                    num(k->info.tau[2]).c_str(), num(k->info.t_end).c_str(), k->info.n_record);
    }
  } else {
    fs::create_directories(o.out_dir, ec);
    for (auto &g : groups) {
      if (o.precision == HEOM_FP64_EXACT) {
        for (Key *k : g) ok &= run_exact(o, *k);
      } else {
        ok &= run_group(o, g);
      }
    }
  }
  for (Key &k : keys) heom_problem_destroy(k.prob);
  return ok ? 0 : 1;
}
