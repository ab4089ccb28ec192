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
