// sa_b200_sys.hpp -- drop-in gpu_sys systems backed by the B200 engine.
//
// b200_2dp / b200_3d replace the reference's gpu_2d / gpu_3d
// (src/gpu_2d.cuh, src/gpu_3d.cuh); b200_2d adds the fully periodic 2D lattice
// of cpu_2d. Each is a gpu_sys (src/gpu_sys.cuh:12-29) over the C ABI in
// sa_b200.h, so the reference's annealing<gpu_sys> and
// parallel_tempering<gpu_sys> templates drive them without change.
//
// Semantics follow the reference: measure() returns the 64-entry float
// vector E + h*M (index j = replica bit j); swap() takes ownership of the
// mask and exchanges the masked replica bits of every spin word; errors are
// reported on std::cerr and execution continues (the reference logs and
// continues, src/gpu_2d.cu:216-220). load_J/save_J use the reference's J file
// format (src/sys_file.cpp:10-110: int dim; long N; Jx[2N]; Jy[2N]; Jz[2N]).
// save()/load() write this engine's own checkpoint record (a length-prefixed
// sa_sys_save blob), not the reference's Philox-state dump.
#pragma once
#include <cstdint>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "sa_b200.h"
#include "sa_gpu_sys.hpp"

class b200_sys : public gpu_sys {
 public:
  b200_sys(int lattice, int L_, double T_, double h_) : lattice_(lattice), L_(L_), h_(h_) {
    report(sa_sys_create(lattice, L_, T_, h_, &sys_), "create");
    if (sys_) sa_sys_get_N(sys_, &N_);
  }
  virtual ~b200_sys() { gpu_free(); }

  void sweep() override { report(sa_sys_sweep(sys_, 1), "sweep"); }
  void set_T(double T_) override { report(sa_sys_set_T(sys_, T_), "set_T"); }
  void set_h(double h) override {
    h_ = h;
    report(sa_sys_set_h(sys_, h), "set_h");
  }
  void set_seed(long long seed_) override { report(sa_sys_set_seed(sys_, (uint64_t)seed_), "set_seed"); }
  vector<float> measure() override {
    vector<float> r(64, 0.f);
    report(sa_sys_measure_float(sys_, r.data()), "measure");
    return r;
  }
  void gpu_free() override {
    if (sys_) {
      sa_sys_destroy(sys_);
      sys_ = nullptr;
    }
  }
  void load_J(string fname) override {
    ifstream f(fname, ios::in | ios::binary);
    int d = 0;
    long n = 0;
    if (!f.is_open()) return warn("cannot open J file \"" + fname + "\"");
    f.read(reinterpret_cast<char*>(&d), sizeof d);
    f.read(reinterpret_cast<char*>(&n), sizeof n);
    if (d != dim() || n != N_) return warn("J file \"" + fname + "\" is for another lattice");
    std::vector<uint64_t> J[3];
    for (int a = 0; a < dim(); ++a) {
      J[a].resize(2 * N_);
      f.read(reinterpret_cast<char*>(J[a].data()), 2 * N_ * sizeof(uint64_t));
    }
    if (!f) return warn("J file \"" + fname + "\" is truncated");
    report(sa_sys_set_J(sys_, J[0].data(), J[1].data(), dim() == 3 ? J[2].data() : nullptr), "load_J");
  }
  void save_J(string fname) override {
    std::vector<uint64_t> J[3];
    for (int a = 0; a < dim(); ++a) J[a].resize(2 * N_);
    if (report(sa_sys_get_J(sys_, J[0].data(), J[1].data(), dim() == 3 ? J[2].data() : nullptr), "save_J"))
      return;
    ofstream f(fname, ios::out | ios::binary);
    if (!f.is_open()) return warn("cannot write J file \"" + fname + "\"");
    int d = dim();
    long n = N_;
    f.write(reinterpret_cast<const char*>(&d), sizeof d);
    f.write(reinterpret_cast<const char*>(&n), sizeof n);
    for (int a = 0; a < dim(); ++a) f.write(reinterpret_cast<const char*>(J[a].data()), 2 * N_ * sizeof(uint64_t));
  }
  void init_J() override { report(sa_sys_init_J(sys_), "init_J"); }
  void init_rand() override { report(sa_sys_init_rand(sys_), "init_rand"); }
  void save_sys(string prefix) override {
    std::vector<uint64_t> s(N_);
    if (report(sa_sys_get_spins(sys_, s.data()), "save_sys")) return;
    const long rows = (dim() == 3) ? (long)L_ * L_ : L_;
    for (int i = 0; i < 64; ++i) {
      std::ostringstream name;
      name << prefix << i << ".pbm";
      ofstream file(name.str());
      file << "P1" << endl << L_ << " " << rows << endl;
      for (long j = 0; j < rows; ++j) {
        for (int k = 0; k < L_; ++k) file << (((s[j * L_ + k] >> i) & 1ULL) ? "1 " : "0 ");
        file << endl;
      }
    }
  }
  long get_N() override { return N_; }
  void swap(gpu_sys* other, std::unique_ptr<spin_t[]> mask) override {
    b200_sys* o = dynamic_cast<b200_sys*>(other);
    if (!o) return warn("swap with a system of another type");
    report(sa_sys_swap(sys_, o->sys_, (uint64_t)mask[0]), "swap");
  }
  ostream& save(ostream& stream) override {
    size_t len = 0;
    if (report(sa_sys_save(sys_, nullptr, 0, &len), "save")) return stream;
    std::vector<char> buf(len);
    if (report(sa_sys_save(sys_, buf.data(), len, &len), "save")) return stream;
    uint64_t n = len;
    stream.write(reinterpret_cast<const char*>(&n), sizeof n);
    return stream.write(buf.data(), (std::streamsize)len);
  }
  istream& load(istream& stream) override {
    uint64_t n = 0;
    stream.read(reinterpret_cast<char*>(&n), sizeof n);
    std::vector<char> buf(n);
    stream.read(buf.data(), (std::streamsize)n);
    if (!stream) {
      warn("checkpoint stream truncated");
      return stream;
    }
    report(sa_sys_load(sys_, buf.data(), n), "load");
    return stream;
  }

  // not part of gpu_sys
  // SA_RNG_MT19937_64: draw from the CPU reference's std::mt19937_64 stream,
  // so results match cpu_2d / cpu_2dp / cpu_3d bit for bit (sa_b200.h).
  void set_rng_mode(int mode) { report(sa_sys_set_rng_mode(sys_, mode), "set_rng_mode"); }
  // cpu_sys::get_T / clone (src/cpu_sys.hpp:28-30), which gpu_sys lacks:
  // parallel_tempering<>::update_T copies a system for an inserted
  // temperature. The copy has its own device allocation and the same
  // spins, couplings, temperature, field and random mode; in mt19937_64 mode
  // its generator is reseeded with 1234 as the reference's copy constructors
  // do (src/cpu_3d.cpp:47-78, src/cpu_2dp.cpp:53-84), in Philox mode it keeps
  // the seed and position.
  double get_T() {
    double t = 0;
    report(sa_sys_get_T(sys_, &t), "get_T");
    return t;
  }
  b200_sys* clone() const {
    b200_sys* c = new b200_sys(lattice_, L_, 1.0, h_);
    size_t len = 0;
    if (sa_sys_save(sys_, nullptr, 0, &len) != SA_OK) return c;
    std::vector<char> buf(len);
    if (sa_sys_save(sys_, buf.data(), len, &len) == SA_OK) c->report(sa_sys_load(c->sys_, buf.data(), len), "clone");
    int mode = SA_RNG_PHILOX;
    if (sa_sys_get_rng_mode(sys_, &mode) == SA_OK && mode == SA_RNG_MT19937_64) {
      size_t rl = 0;
      if (sa_sys_save_reference(sys_, nullptr, 0, &rl) == SA_OK) {
        std::vector<char> rb(rl);
        if (sa_sys_save_reference(sys_, rb.data(), rl, &rl) == SA_OK)
          c->report(sa_sys_load_reference(c->sys_, rb.data(), rl), "clone");
      }
      c->report(sa_sys_set_seed(c->sys_, 1234), "clone");
    }
    return c;
  }
  // runs the system's work on `stream` (a cudaStream_t)
  void set_stream(void* stream) { report(sa_sys_set_stream(sys_, stream), "set_stream"); }
  // colour of each sweep's first half-sweep (sa_sys_set_first_colour)
  void set_first_colour(int c) { report(sa_sys_set_first_colour(sys_, c), "set_first_colour"); }
  // replicas per system (64 here; 128 for b200_sys128)
  static constexpr int replicas() { return 64; }
  sa_system_t handle() const { return sys_; }
  int lattice() const { return lattice_; }
  void get_spins(uint64_t* s) { report(sa_sys_get_spins(sys_, s), "get_spins"); }
  int dim() const { return lattice_ == SA_LATTICE_3D ? 3 : 2; }

 protected:
  // Reference error convention: report and continue. Returns true on error.
  bool report(int status, const char* what) {
    if (status == SA_OK) return false;
    std::cerr << "Error: b200 " << what << ": " << sa_status_string(status) << " (" << sa_last_error() << ")"
              << std::endl;
    return true;
  }
  void warn(const std::string& msg) { std::cerr << "Warning: b200: " << msg << std::endl; }

  sa_system_t sys_ = nullptr;
  int lattice_;
  int L_;
  long N_ = 0;
  double h_;
};

// gpu_2d replacement: square lattice, open in x, periodic in y.
class b200_2dp : public b200_sys {
 public:
  b200_2dp(int L, double T, double h) : b200_sys(SA_LATTICE_2D_OPEN_X, L, T, h) {}
};

// cpu_2d's lattice on the GPU: square, periodic in x and y.
class b200_2d : public b200_sys {
 public:
  b200_2d(int L, double T, double h) : b200_sys(SA_LATTICE_2D, L, T, h) {}
};

// gpu_3d replacement: cubic, periodic.
class b200_3d : public b200_sys {
 public:
  b200_3d(int L, double T, double h) : b200_sys(SA_LATTICE_3D, L, T, h) {}
};

// The reference GPU systems' own shape: 128 replicas per system. gpu_2d and
// gpu_3d keep two lattices s1, s2 and update every site of one from the other
// (src/gpu_2d.cu:109-120, src/gpu_3d.cu:98-110); that carries two
// configurations, A = (s1 on colour-0 sites, s2 on colour-1 sites), whose
// sweep updates colour 0 then colour 1, and B, the complement, which updates
// colour 1 first. b200_sys128 holds them as two systems of this engine with
// the same couplings, A in the usual order and B with first colour 1 (B's
// initial spins come from a counter range of its own). measure() returns A's
// 64 values then B's (src/gpu_2d.cu:196-205); swap() takes one mask word for
// each (src/parallel_tempering.hpp:143-149 makes E.size()/64 words).
// Philox mode only; there is no CPU counterpart of the two-lattice trick.
class b200_sys128 : public gpu_sys {
 public:
  b200_sys128(int lattice, int L, double T, double h) : a_(lattice, L, T, h), b_(lattice, L, T, h), L_(L) {
    b_.set_first_colour(1);
  }
  void sweep() override {
    a_.sweep();
    b_.sweep();
  }
  void set_T(double T) override {
    a_.set_T(T);
    b_.set_T(T);
  }
  void set_h(double h) override {
    a_.set_h(h);
    b_.set_h(h);
  }
  void set_seed(long long s) override {
    a_.set_seed(s);
    b_.set_seed(s);
  }
  vector<float> measure() override {
    vector<float> r = a_.measure(), rb = b_.measure();
    r.insert(r.end(), rb.begin(), rb.end());
    return r;
  }
  void gpu_free() override {
    a_.gpu_free();
    b_.gpu_free();
  }
  void load_J(string fname) override {
    a_.load_J(fname);
    b_.load_J(fname);
  }
  void save_J(string fname) override { a_.save_J(fname); }
  void init_J() override {
    a_.init_J();
    b_.init_J();
  }
  void init_rand() override {
    a_.init_rand();
    b_.init_rand();
  }
  // PBM images: replicas 0..63 from A, 64..127 from B
  void save_sys(string prefix) override {
    const long N = a_.get_N();
    const long rows = (a_.dim() == 3) ? (long)L_ * L_ : L_;
    for (int half = 0; half < 2; ++half) {
      std::vector<uint64_t> s(N);
      (half ? b_ : a_).get_spins(s.data());
      for (int i = 0; i < 64; ++i) {
        std::ostringstream name;
        name << prefix << (64 * half + i) << ".pbm";
        ofstream file(name.str());
        file << "P1" << endl << L_ << " " << rows << endl;
        for (long j = 0; j < rows; ++j) {
          for (int k = 0; k < L_; ++k) file << (((s[j * L_ + k] >> i) & 1ULL) ? "1 " : "0 ");
          file << endl;
        }
      }
    }
  }
  long get_N() override { return a_.get_N(); }
  void swap(gpu_sys* other, std::unique_ptr<spin_t[]> mask) override {
    b200_sys128* o = dynamic_cast<b200_sys128*>(other);
    if (!o) {
      std::cerr << "Warning: b200: swap with a system of another type" << std::endl;
      return;
    }
    std::unique_ptr<spin_t[]> ma(new spin_t[1]), mb(new spin_t[1]);
    ma[0] = mask[0];
    mb[0] = mask[1];
    a_.swap(&o->a_, std::move(ma));
    b_.swap(&o->b_, std::move(mb));
  }
  ostream& save(ostream& stream) override {
    a_.save(stream);
    return b_.save(stream);
  }
  istream& load(istream& stream) override {
    a_.load(stream);
    return b_.load(stream);
  }
  // not part of gpu_sys
  double get_T() { return a_.get_T(); }
  b200_sys128* clone() const {
    b200_sys128* c = new b200_sys128(a_.lattice(), L_, 1.0, 0.0);
    std::stringstream ss;
    const_cast<b200_sys&>(a_).save(ss);
    const_cast<b200_sys&>(b_).save(ss);
    c->load(ss);
    return c;
  }
  void set_stream(void* stream) {
    a_.set_stream(stream);
    b_.set_stream(stream);
  }
  void set_rng_mode(int mode) {
    if (mode != SA_RNG_PHILOX) std::cerr << "Error: b200: the two-lattice systems run in Philox mode only" << std::endl;
  }
  static constexpr int replicas() { return 128; }
  b200_sys& first() { return a_; }
  b200_sys& second() { return b_; }

 private:
  b200_sys a_, b_;
  int L_;
};

// gpu_2d's shape (open in x, periodic in y) and gpu_3d's, 128 replicas each
class b200_2dp_128 : public b200_sys128 {
 public:
  b200_2dp_128(int L, double T, double h) : b200_sys128(SA_LATTICE_2D_OPEN_X, L, T, h) {}
};
class b200_3d_128 : public b200_sys128 {
 public:
  b200_3d_128(int L, double T, double h) : b200_sys128(SA_LATTICE_3D, L, T, h) {}
};
