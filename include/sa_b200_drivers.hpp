// sa_b200_drivers.hpp -- the annealing and parallel-tempering drivers in C++,
// for programs that do not take the reference's own templates.
//
// sa_b200::annealing<System> and sa_b200::parallel_tempering<System> have the
// member functions, arguments and results of the reference's
// annealing<system> (src/annealing.hpp:10-29) and parallel_tempering<system>
// (src/parallel_tempering.hpp:17-52). The exchange generator is the engine's
// sa_pt_gen (std::mt19937(123) with the template's two distributions), the
// exchange test sa_pt_mask (src/parallel_tempering.hpp:141-162), so a run
// makes the reference's decisions. save()/load() write and read the
// template's checkpoint stream (src/parallel_tempering.hpp:280-377) with each
// system's own save()/load() record.
//
// System: sweep(), measure() -> std::vector<float> (64 values per 64
// replicas), set_T(double), swap(System*, std::unique_ptr<spin_t[]>) with one
// mask word per 64 replicas, init_rand(), save(std::ostream&) and
// load(std::istream&); update_T() also needs clone() -> System* (the engine's
// b200_sys has it; gpu_sys itself does not). Errors follow the reference's
// convention: a message on std::cerr, and the run continues.
#ifndef SA_B200_DRIVERS_HPP
#define SA_B200_DRIVERS_HPP

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "sa_b200.h"

namespace sa_b200 {

typedef unsigned long long spin_t;

enum print_select { PRINT_E, PRINT_MIN };

// `name` with every '%' replaced by `with` (the reference uses
// std::regex_replace on the first and every later '%').
inline std::string replace_percent(const std::string& name, const std::string& with) {
  std::string out;
  for (char c : name) {
    if (c == '%') out += with;
    else out += c;
  }
  return out;
}

template <class System>
class annealing {
 public:
  annealing(double T_s, int steps_, double alfa_, System* S, std::ostream& file_ = std::cout)
      : T(T_s), alfa(alfa_), steps(steps_), file(&file_), sys(S) {
    sys->set_T(T);
  }
  // steps sweeps, a measurement every `stride` (running maximum of -H per
  // replica), then T *= alfa (src/annealing.hpp:67-100)
  void step(int stride, print_select select = PRINT_E) {
    for (int i = 0; i < steps; ++i) {
      sys->sweep();
      if (stride != 0 && i % stride == 0) {
        result = sys->measure();
        if (min_E.empty()) min_E = result;
        if (min_E.size() == result.size()) {
          for (size_t j = 0; j < min_E.size(); ++j) min_E[j] = std::max(result[j], min_E[j]);
        } else {
          std::cerr << "Error: min_E and result are not the same size" << std::endl;
        }
        if (select == PRINT_E) print(select);
      }
    }
    T = T * alfa;
    sys->set_T(T);
  }
  void print(print_select select) {
    const std::vector<float>& data = (select == PRINT_MIN) ? min_E : result;
    for (float v : data) (*file) << v << "\t";
    (*file) << std::endl;
  }
  double get_T() const { return T; }
  // sets T and clears the running maximum (src/annealing.hpp:129-139)
  void set_T(double T_s) {
    T = T_s;
    min_E.clear();
  }
  const std::vector<float>& get_min_E() const { return min_E; }

 private:
  double T, alfa;
  int steps;
  std::ostream* file;
  System* sys;
  std::vector<float> min_E, result;
};

template <class System>
class parallel_tempering {
 public:
  parallel_tempering(std::vector<System*>& sys_, const std::vector<double>& T_, long steps_,
                     const std::string& filename)
      : sys(sys_), T(T_), steps(steps_), fname(filename) {
    if (T.size() != sys.size() || T.size() < 2)
      std::cerr << "Error: size difference : sys " << sys.size() << " T " << T.size() << std::endl;
    std::sort(T.begin(), T.end());
    num_sum.assign(T.size() > 0 ? T.size() - 1 : 0, 0.0);
    num_n.assign(num_sum.size(), 0);
    E.assign(T.size(), std::vector<float>());
    if (sa_pt_gen_create((int)std::max<size_t>(T.size(), 2), &gen) != SA_OK) gen = nullptr;
    for (size_t i = 0; i < T.size() && i < sys.size(); ++i) sys[i]->set_T(T[i]);
  }
  ~parallel_tempering() {
    if (gen) sa_pt_gen_destroy(gen);
  }
  parallel_tempering(const parallel_tempering&) = delete;
  parallel_tempering& operator=(const parallel_tempering&) = delete;

  // `steps` sweeps of every slot with measurements, then one exchange attempt
  // between a random adjacent pair (src/parallel_tempering.hpp:81-115)
  void step(int stride) {
    for (long i = 0; i < steps; ++i) {
      for (size_t j = 0; j < T.size(); ++j) {
        sys[j]->sweep();
        if ((stride != 0 && i % stride == 0) || i == steps - 1) E[j] = sys[j]->measure();
      }
      if (stride != 0 && i % stride == 0) {
        print(PRINT_E);
      } else if (stride == 0) {
        if (E_min.empty()) E_min = E[0];
        for (size_t j = 0; j < E_min.size() && j < E[0].size(); ++j) E_min[j] = std::max(E[0][j], E_min[j]);
      }
    }
    int32_t pair = 0;
    double r = 0;
    sa_pt_gen_next(gen, 1, &pair, &r);
    last_pair = pair;
    sys[pair]->swap(sys[pair + 1], creat_mask(pair, r));
  }

  void print(print_select select) {
    open_files(select, false);
    if (select == PRINT_E) {
      for (size_t i = 0; i < T.size(); ++i) {
        for (float v : E[i]) (*files[i]) << v << "\t";
        (*files[i]) << "\n";
      }
    } else {
      for (float v : E_min) (*file_E_min) << v << "\t";
      (*file_E_min) << std::endl;
    }
  }
  void print_swap(std::ostream& f) {
    for (size_t i = 0; i + 1 < T.size(); ++i) f << T[i] << " -> " << T[i + 1] << "\t: " << acceptance(i) << "\n";
  }
  void set_info(const std::string& info, print_select select) {
    open_files(select, false);
    if (select == PRINT_E) {
      for (auto& f : files) (*f) << info;
    } else {
      (*file_E_min) << info;
    }
  }
  // E_min to 0 and new random spins in every slot; the acceptance counters
  // stay (the reference's accumulator::reset is a no-op,
  // src/accumulator.hpp:36-38)
  void reset() {
    std::fill(E_min.begin(), E_min.end(), 0.0f);
    for (System* s : sys) s->init_rand();
  }
  std::vector<float> get_E_min() const { return E_min; }
  double acceptance(size_t i) const { return num_sum[i] != 0 ? num_sum[i] / (double)num_n[i] : 0.0; }
  int get_last_pair() const { return last_pair; }
  const std::vector<double>& get_T() const { return T; }

  // the template's checkpoint stream (src/parallel_tempering.hpp:280-318)
  std::ostream& save(std::ostream& stream) {
    put(stream, steps);
    put(stream, print_E);
    put(stream, print_min);
    size_t glen = 0;
    sa_pt_gen_save(gen, nullptr, 0, &glen);
    std::vector<char> g(glen);
    sa_pt_gen_save(gen, g.data(), glen, &glen);
    stream.write(g.data(), (std::streamsize)glen);
    put(stream, fname.size());
    stream.write(fname.data(), (std::streamsize)fname.size());
    put(stream, T.size());
    stream.write(reinterpret_cast<const char*>(T.data()), (std::streamsize)(T.size() * sizeof(double)));
    put(stream, E_min.size());
    stream.write(reinterpret_cast<const char*>(E_min.data()), (std::streamsize)(E_min.size() * sizeof(float)));
    put(stream, num_sum.size());
    for (size_t i = 0; i < num_sum.size(); ++i) {
      put(stream, num_sum[i]);
      put(stream, num_n[i]);
    }
    put(stream, E.size());
    for (size_t i = 0; i < E.size(); ++i) {
      put(stream, E[i].size());
      stream.write(reinterpret_cast<const char*>(E[i].data()), (std::streamsize)(E[i].size() * sizeof(float)));
      sys[i]->save(stream);
    }
    return stream;
  }
  // reads save()'s stream (src/parallel_tempering.hpp:320-377); the file
  // name read is kept (the reference's reader drops it, src/bin_io.cpp:3-8)
  std::istream& load(std::istream& stream) {
    files.clear();
    file_E_min.reset();
    get(stream, steps);
    bool pe = false, pm = false;
    get(stream, pe);
    get(stream, pm);
    size_t glen = 0;
    sa_pt_gen_save(gen, nullptr, 0, &glen);
    std::vector<char> g(glen);
    stream.read(g.data(), (std::streamsize)glen);
    if (stream) sa_pt_gen_load(gen, g.data(), glen);
    size_t n = 0;
    get(stream, n);
    fname.assign(n, '\0');
    if (n) stream.read(&fname[0], (std::streamsize)n);
    get(stream, n);
    T.assign(n, 0.0);
    stream.read(reinterpret_cast<char*>(T.data()), (std::streamsize)(n * sizeof(double)));
    print_E = print_min = false;
    if (pe) open_files(PRINT_E, true);
    if (pm) open_files(PRINT_MIN, true);
    get(stream, n);
    E_min.assign(n, 0.0f);
    stream.read(reinterpret_cast<char*>(E_min.data()), (std::streamsize)(n * sizeof(float)));
    get(stream, n);
    num_sum.assign(n, 0.0);
    num_n.assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
      get(stream, num_sum[i]);
      get(stream, num_n[i]);
    }
    get(stream, n);
    if (n != sys.size()) {
      std::cerr << "Error: checkpoint holds " << n << " systems, the driver has " << sys.size() << std::endl;
      stream.setstate(std::ios::failbit);
      return stream;
    }
    E.assign(n, std::vector<float>());
    for (size_t i = 0; i < n; ++i) {
      size_t m = 0;
      get(stream, m);
      E[i].assign(m, 0.0f);
      stream.read(reinterpret_cast<char*>(E[i].data()), (std::streamsize)(m * sizeof(float)));
      sys[i]->load(stream);
    }
    if (!stream) std::cerr << "Error: checkpoint stream truncated" << std::endl;
    return stream;
  }
  // after every pair whose acceptance is below 0.3, insert the mean of its
  // two temperatures carried by a copy of the pair's upper system
  // (src/parallel_tempering.hpp:384-413)
  void update_T() {
    for (size_t i = 0; i < num_sum.size(); i++) {
      if (acceptance(i) < 0.3) {
        i++;
        num_sum.insert(num_sum.begin() + i, 0.0);
        num_n.insert(num_n.begin() + i, 0);
        const double t = (T[i] + T[i - 1]) / 2.0;
        T.insert(T.begin() + i, t);
        E.insert(E.begin() + i, std::vector<float>());
        System* c = sys[i]->clone();
        sys.insert(sys.begin() + i, c);
        owned.emplace_back(c);
        sys[i]->set_T(T[i]);
        if (print_E)
          files.insert(files.begin() + i, std::unique_ptr<std::ofstream>(new std::ofstream(
                                              replace_percent(fname, "T" + std::to_string(T[i])), std::ios::out)));
        sa_pt_gen_widen(gen);
      }
    }
  }
  // the systems in temperature order (update_T adds copies it owns)
  const std::vector<System*>& systems() const { return sys; }

 private:
  template <class V>
  static void put(std::ostream& s, const V& v) {
    s.write(reinterpret_cast<const char*>(&v), sizeof v);
  }
  template <class V>
  static void get(std::istream& s, V& v) {
    s.read(reinterpret_cast<char*>(&v), sizeof v);
  }
  // one mask word per 64 replicas, bit j of word w for replica 64w+j
  std::unique_ptr<spin_t[]> creat_mask(int i, double r) {
    const size_t words = E[i].size() / 64;
    std::unique_ptr<spin_t[]> mask(new spin_t[std::max<size_t>(words, 1)]());
    int a = 0;
    for (size_t w = 0; w < words; ++w) {
      mask[w] = sa_pt_mask(E[i].data() + 64 * w, E[i + 1].data() + 64 * w, T[i], T[i + 1], r);
      a += __builtin_popcountll(mask[w]);
    }
    num_sum[i] += a / 64.0;
    num_n[i] += 1;
    return mask;
  }
  void open_files(print_select select, bool append) {
    const std::ios_base::openmode mode = append ? std::ios_base::app : std::ios_base::out;
    if (select == PRINT_E && !print_E) {
      for (double t : T)
        files.emplace_back(new std::ofstream(replace_percent(fname, "T" + std::to_string(t)), mode));
      print_E = true;
    } else if (select == PRINT_MIN && !print_min) {
      file_E_min.reset(new std::ofstream(replace_percent(fname, "E_min"), mode));
      print_min = true;
    }
  }

  std::vector<System*> sys;
  std::vector<double> T;
  std::vector<std::vector<float>> E;
  std::vector<float> E_min;
  std::vector<double> num_sum;
  std::vector<long long> num_n;
  long steps;
  std::string fname;
  bool print_E = false, print_min = false;
  std::vector<std::unique_ptr<std::ofstream>> files;
  std::unique_ptr<std::ofstream> file_E_min;
  sa_pt_gen_t gen = nullptr;
  int last_pair = -1;
  std::vector<std::unique_ptr<System>> owned;
};

}  // namespace sa_b200

#endif  // SA_B200_DRIVERS_HPP
