// ref_driver.cpp -- C entry points around the reference's OWN CPU classes.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle). Compiled together with the
// unmodified reference sources cpu_2d.cpp, cpu_2dp.cpp, cpu_3d.cpp,
// Logging.cpp, bin_io.cpp, sys_file.cpp (read in place from the reference
// tree by oracle/Makefile; nothing is copied) into oracle/_ref/libsa_ref.so.
// It exists so the oracle's restatement (sa_oracle.cpp, MT mode) can be
// compared bit for bit with the reference itself, and so bench.py can time
// the reference CPU path as its CPU baseline.
//
// State is read back through the reference's own save() stream
// (src/cpu_2dp.cpp:444-456, src/cpu_3d.cpp:449-461). Parallel-tempering
// decisions are observed by wrapping each system in a forwarding cpu_sys that
// records the (pair, mask) the reference template passes to swap()
// (src/parallel_tempering.hpp:112-114).
#include <cstdint>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <omp.h>

#include "annealing.hpp"
#include "cpu_2d.hpp"
#include "cpu_2dp.hpp"
#include "cpu_3d.hpp"
#include "parallel_tempering.hpp"

namespace {

struct RefSys {
  cpu_sys* sys;
  int kind;  // 0: cpu_2d (periodic), 1: cpu_2dp (open x), 2: cpu_3d
  int L;
};

struct SwapLog {
  std::vector<int> pair;
  std::vector<spin_t> mask;
  std::vector<double> T;  // temperature of the pair's lower system
};

class spy_sys : public cpu_sys {
 public:
  cpu_sys* in;
  int id;
  SwapLog* log;
  spy_sys(cpu_sys* s, int i, SwapLog* l) : in(s), id(i), log(l) {}
  void set_seed(long se) override { in->set_seed(se); }
  void init_rand() override { in->init_rand(); }
  void init_order() override { in->init_order(); }
  void init_J() override { in->init_J(); }
  void load_J(string f) override { in->load_J(f); }
  void save_J(string f) override { in->save_J(f); }
  void sweep() override { in->sweep(); }
  void set_T(double T) override { in->set_T(T); }
  vector<float> measure() override { return in->measure(); }
  void save_sys(string p) override { in->save_sys(p); }
  long get_N() override { return in->get_N(); }
  double get_T() override { return in->get_T(); }
  void swap(cpu_sys* other, std::unique_ptr<spin_t[]> mask) override {
    log->pair.push_back(id);
    log->mask.push_back(mask[0]);
    log->T.push_back(in->get_T());
    in->swap(static_cast<spy_sys*>(other)->in, std::move(mask));
  }
  ostream& save(ostream& s) override { return in->save(s); }
  istream& load(istream& s) override { return in->load(s); }
  cpu_sys* clone() const override { return new spy_sys(in->clone(), id, log); }
};

struct RefPT {
  SwapLog log;
  std::vector<cpu_sys*> spies;
  std::string fname;
  std::unique_ptr<parallel_tempering<cpu_sys>> pt;
};

}  // namespace

extern "C" {

// OpenMP threads of the calling host thread's parallel regions (the PT
// template's loop over slots, src/parallel_tempering.hpp:86). The CPU baseline
// runs one instance per host thread with 1, so the cores go to instances.
void ref_omp_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

void* ref_sys_new(int kind, int L, double T, double h) {
  RefSys* r = new RefSys();
  r->kind = kind;
  r->L = L;
  if (kind == 0) r->sys = new cpu_2d(L, T, h);
  else if (kind == 1) r->sys = new cpu_2dp(L, T, h);
  else r->sys = new cpu_3d(L, T, h);
  return r;
}
void ref_sys_free(void* p) {
  RefSys* r = (RefSys*)p;
  delete r->sys;
  delete r;
}
void ref_set_seed(void* p, long seed) { ((RefSys*)p)->sys->set_seed(seed); }
void ref_init_J(void* p) { ((RefSys*)p)->sys->init_J(); }
void ref_init_rand(void* p) { ((RefSys*)p)->sys->init_rand(); }
void ref_init_order(void* p) { ((RefSys*)p)->sys->init_order(); }
void ref_set_T(void* p, double T) { ((RefSys*)p)->sys->set_T(T); }
void ref_sweep(void* p, long n) {
  RefSys* r = (RefSys*)p;
  for (long i = 0; i < n; ++i) r->sys->sweep();
}
void ref_measure(void* p, float* out64) {
  std::vector<float> v = ((RefSys*)p)->sys->measure();
  for (size_t i = 0; i < v.size() && i < 64; ++i) out64[i] = v[i];
}
long ref_get_N(void* p) { return ((RefSys*)p)->sys->get_N(); }

// Spins and the reference-layout couplings, parsed from save():
// int L, double T, double h, s[N], Jx[2N], Jy[2N], (Jz[2N]), generator state...
void ref_get_state(void* p, uint64_t* s, uint64_t* jx, uint64_t* jy, uint64_t* jz) {
  RefSys* r = (RefSys*)p;
  std::stringstream ss;
  r->sys->save(ss);
  std::string b = ss.str();
  long N = r->sys->get_N();
  size_t off = sizeof(int) + 2 * sizeof(double);
  memcpy(s, b.data() + off, N * 8);
  off += N * 8;
  memcpy(jx, b.data() + off, 2 * N * 8);
  off += 2 * N * 8;
  memcpy(jy, b.data() + off, 2 * N * 8);
  off += 2 * N * 8;
  if (r->kind == 2 && jz) memcpy(jz, b.data() + off, 2 * N * 8);
}

void ref_swap(void* a, void* b, uint64_t mask) {
  std::unique_ptr<spin_t[]> m(new spin_t[1]);
  m[0] = mask;
  ((RefSys*)a)->sys->swap(((RefSys*)b)->sys, std::move(m));
}

// parallel_tempering<cpu_sys> over the given systems (ownership stays with the
// caller). stride 0 keeps the template from opening output files.
void* ref_pt_new(void** systems, const double* T, int n, long steps) {
  RefPT* r = new RefPT();
  r->fname = "unused_%";
  for (int i = 0; i < n; ++i)
    r->spies.push_back(new spy_sys(((RefSys*)systems[i])->sys, i, &r->log));
  std::vector<double> Tv(T, T + n);
  r->pt.reset(new parallel_tempering<cpu_sys>(r->spies, Tv, steps, r->fname));
  return r;
}
void ref_pt_step(void* p, int stride, int* pair, uint64_t* mask) {
  RefPT* r = (RefPT*)p;
  r->pt->step(stride);
  *pair = r->log.pair.back();
  *mask = r->log.mask.back();
}
// The lower temperature of the last exchange's pair (after update_T the
// systems' creation indices no longer name pairs).
double ref_pt_last_T(void* p) { return ((RefPT*)p)->log.T.back(); }
void ref_pt_update_T(void* p) { ((RefPT*)p)->pt->update_T(); }
// parallel_tempering<>::save / load streams (the .tempsys checkpoint).
long ref_pt_save(void* p, char* buf, long cap) {
  std::stringstream ss;
  ((RefPT*)p)->pt->save(ss);
  std::string b = ss.str();
  if (buf && cap >= (long)b.size()) memcpy(buf, b.data(), b.size());
  return (long)b.size();
}
void ref_pt_load(void* p, const char* buf, long len) {
  std::stringstream ss(std::string(buf, (size_t)len));
  ((RefPT*)p)->pt->load(ss);
}
int ref_pt_print_swap(void* p, char* buf, int len) {
  std::stringstream ss;
  ((RefPT*)p)->pt->print_swap(ss);
  std::string s = ss.str();
  int n = (int)std::min<size_t>(s.size(), (size_t)len - 1);
  memcpy(buf, s.data(), n);
  buf[n] = 0;
  return n;
}
void ref_pt_free(void* p) {
  RefPT* r = (RefPT*)p;
  r->pt.reset();
  for (cpu_sys* s : r->spies) delete static_cast<spy_sys*>(s);
  delete r;
}

// annealing<cpu_sys>: nsteps calls of step(stride, PRINT_MIN), then the running
// maximum printed by print(PRINT_MIN) is parsed back into min_E.
void ref_anneal_run(void* p, double T0, double alfa, int nsteps, int sweeps, int stride,
                    float* min_E) {
  std::stringstream out;
  annealing<cpu_sys> a(T0, sweeps, alfa, ((RefSys*)p)->sys, out);
  for (int k = 0; k < nsteps; ++k) a.step(stride, PRINT_MIN);
  std::stringstream res;
  std::ostream* keep = &res;
  (void)keep;
  annealing<cpu_sys>* ap = &a;
  // print() writes to the stream given at construction
  ap->print(PRINT_MIN);
  std::string line = out.str();
  std::stringstream in(line);
  for (int j = 0; j < 64; ++j) in >> min_E[j];
}

// The reference object's own J file writer and reader (cpu_2dp::save_J /
// load_J -> save_J_2d / load_J_2d, cpu_3d -> *_3d; src/sys_file.cpp:10-110).
void ref_save_J(void* p, const char* fname) { ((RefSys*)p)->sys->save_J(std::string(fname)); }
void ref_load_J(void* p, const char* fname) { ((RefSys*)p)->sys->load_J(std::string(fname)); }

// The reference object's own save() / load() byte stream (its checkpoint
// record), for comparing this engine's record with it.
long ref_save(void* p, char* buf, long cap) {
  RefSys* r = (RefSys*)p;
  std::stringstream ss;
  r->sys->save(ss);
  std::string b = ss.str();
  if (buf && cap >= (long)b.size()) memcpy(buf, b.data(), b.size());
  return (long)b.size();
}
void ref_load(void* p, const char* buf, long len) {
  RefSys* r = (RefSys*)p;
  std::stringstream ss(std::string(buf, (size_t)len));
  r->sys->load(ss);
}

}  // extern "C"
