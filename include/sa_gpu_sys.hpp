// sa_gpu_sys.hpp -- the gpu_sys system interface (src/gpu_sys.cuh:12-29).
//
// The abstract class the reference's drivers (annealing<system>,
// parallel_tempering<system>) program against. Code that already has the
// reference's own gpu_sys.cuh defines SA_HAVE_REFERENCE_GPU_SYS and includes
// that header first; the shim in sa_b200_sys.hpp then derives from it, so the
// reference templates drive this engine unchanged. Otherwise this declaration
// (same members, same signatures) stands in for it.
#pragma once
#ifndef SA_HAVE_REFERENCE_GPU_SYS
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

using namespace std;

typedef unsigned long long spin_t;

class gpu_sys {
 public:
  virtual void sweep() = 0;
  virtual void set_T(double T_) = 0;
  virtual void set_h(double h_) = 0;
  virtual void set_seed(long long seed_) = 0;
  virtual vector<float> measure() = 0;
  virtual void gpu_free() = 0;
  virtual void load_J(string fname) = 0;
  virtual void save_J(string fname) = 0;
  virtual void init_J() = 0;
  virtual void init_rand() = 0;
  virtual void save_sys(string prefix) = 0;
  virtual long get_N() = 0;
  virtual void swap(gpu_sys* sys, std::unique_ptr<spin_t[]> mask) = 0;
  virtual ostream& save(ostream& stream) = 0;
  virtual istream& load(istream& stream) = 0;
};
#endif
