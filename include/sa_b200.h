/*
 * sa_b200.h -- C ABI of the B200 multispin-coded Ising spin-glass engine.
 *
 * One "system" is one lattice carrying 64 replicas, one bit each, in a 64-bit
 * word per site: the reference's gpu_sys / cpu_sys object
 * (src/gpu_sys.cuh:12-29, src/cpu_sys.hpp:12-31). Every entry point:
 *   - is extern "C", takes plain pointers and sizes, and never throws;
 *   - returns an int status (SA_OK == 0); sa_last_error() gives a message for
 *     the calling thread;
 *   - is safe to call concurrently on DISTINCT handles.
 * Host buffers use the reference's row-major layout (site i = x + L*y + L*L*z)
 * and its duplicated coupling layout J?[2N] (J?[2i] = bond to the -x/-y/-z
 * neighbour, J?[2i+1] = bond to the +x/+y/+z neighbour). Energies cross the
 * ABI as exact integers per replica bit j (index j = bit j, which is also the
 * index the reference's float vectors use).
 *
 * Random numbers follow the reference GPU schedule (src/random.cu:15-35,
 * src/device_2d.cu:96-97): site i draws from Philox4x32-10 stream
 * (key = seed, subsequence = i); every site consumes one draw per half-sweep,
 * so a system's whole RNG state is (seed, draw counter).
 */
#ifndef SA_B200_H
#define SA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
enum {
  SA_OK = 0,
  SA_ERR_INVALID = 1,      /* bad argument (null pointer, size, range) */
  SA_ERR_ODD_L = 2,        /* L must be even (checkerboard colouring) */
  SA_ERR_CUDA = 3,         /* a CUDA runtime call failed */
  SA_ERR_NO_DEVICE = 4,    /* no CUDA device / extension unusable */
  SA_ERR_MISMATCH = 5,     /* two systems of different shape */
  SA_ERR_J_INCONSISTENT = 6, /* duplicated coupling words disagree */
  SA_ERR_BUFFER = 7,       /* caller buffer too small / bad checkpoint */
  SA_ERR_BUDGET = 8,       /* memory budget exceeded */
  SA_ERR_TIMEOUT = 9,      /* a bounded device-side wait gave up */
  SA_ERR_UNSUPPORTED = 10  /* valid request this build does not handle */
};

/* lattice kinds (the reference classes they replace) */
enum {
  SA_LATTICE_2D = 0,        /* cpu_2d: square, periodic in x and y */
  SA_LATTICE_2D_OPEN_X = 1, /* cpu_2dp / gpu_2d: open in x, periodic in y */
  SA_LATTICE_3D = 2         /* cpu_3d / gpu_3d: cubic, periodic */
};

/* Random-number modes (sa_sys_set_rng_mode). */
enum {
  SA_RNG_PHILOX = 0,     /* the GPU reference's cuRAND Philox schedule (default) */
  SA_RNG_MT19937_64 = 1  /* the CPU reference's std::mt19937_64 stream */
};

typedef struct sa_system* sa_system_t;

/* Last error message of the calling thread ("" if none). */
const char* sa_last_error(void);
/* Static description of a status code. */
const char* sa_status_string(int status);
/* Library version string. */
const char* sa_version(void);

/* ---- single systems: the gpu_sys boundary ----------------------------------- */

/* Constructor: gpu_2d(L,T,h) src/gpu_2d.cu:23-84, gpu_3d(L,T,h) src/gpu_3d.cu:20-77.
 * Allocates spins and couplings on the current device, keys the generator with
 * seed 1234 (src/gpu_2d.cu:47) and zeroes spins and couplings. */
int sa_sys_create(int lattice, int L, double T, double h, sa_system_t* out);
/* gpu_free() + delete: src/gpu_2d.cu:90-107. */
int sa_sys_destroy(sa_system_t sys);
/* Run this system's work on `stream` (a cudaStream_t; NULL = the system's own). */
int sa_sys_set_stream(sa_system_t sys, void* stream);
/* set_T: src/gpu_2d.cu:122-147 (Boltzmann table -> integer thresholds). */
int sa_sys_set_T(sa_system_t sys, double T);
/* set_h: src/gpu_2d.cu:149-173. */
int sa_sys_set_h(sa_system_t sys, double h);
int sa_sys_get_T(sa_system_t sys, double* T);
/* set_seed: src/gpu_3d.cu:205-210 (re-keys every site's stream, draw counter 0). */
int sa_sys_set_seed(sa_system_t sys, uint64_t seed);
/* init_J: src/gpu_2d.cu:247-257 (2*dim draws per site -> own bond words). */
int sa_sys_init_J(sa_system_t sys);
/* init_rand: src/gpu_2d.cu:259-264. Counter-based here: site i takes Philox
 * block (epoch, 0, i, 2^31 | i>>32) of key seed; each call advances the epoch. */
int sa_sys_init_rand(sa_system_t sys);
/* init_order: src/cpu_2dp.cpp:296-301 (all spins up). */
int sa_sys_init_order(sa_system_t sys);
/* load_J / save_J data path (src/gpu_2d.cu:213-244): host arrays of 2N words
 * each, jz ignored for 2D. set_J rejects duplicated words that disagree. */
int sa_sys_set_J(sa_system_t sys, const uint64_t* jx, const uint64_t* jy, const uint64_t* jz);
int sa_sys_get_J(sa_system_t sys, uint64_t* jx, uint64_t* jy, uint64_t* jz);
/* Spins, host row-major, N words. */
int sa_sys_set_spins(sa_system_t sys, const uint64_t* s);
int sa_sys_get_spins(sa_system_t sys, uint64_t* s);
/* sweep(): src/gpu_2d.cu:109-120 -- here `nsweeps` full sweeps, two
 * half-sweep launches each, asynchronous on the system's stream. */
int sa_sys_sweep(sa_system_t sys, long nsweeps);
/* measure(): src/gpu_2d.cu:176-211. E[j] = sum over bonds of (+1 satisfied,
 * -1 not), M[j] = sum over sites of (+1 up, -1 down), j = replica bit. Host
 * outputs; synchronises the system's stream. */
int sa_sys_measure(sa_system_t sys, int64_t* E, int64_t* M);
/* The reference's float vector: out[j] = (float)(E[j] + h*M[j]). */
int sa_sys_measure_float(sa_system_t sys, float* out64);
/* Device-side measure into DEVICE arrays E[64], M[64] (int64), asynchronous. */
int sa_sys_measure_async(sa_system_t sys, int64_t* d_E, int64_t* d_M);
/* swap(sys, mask): src/gpu_2d.cu:305-324 -- bit-masked exchange of all spin
 * words between two systems of the same shape (src/tools_inline.hpp:4-9). */
int sa_sys_swap(sa_system_t a, sa_system_t b, uint64_t mask);
/* get_N: src/gpu_2d.cu:301-303. */
int sa_sys_get_N(sa_system_t sys, long* N);
/* Random-number source of a system.
 * SA_RNG_PHILOX (default): the GPU reference's schedule, cuRAND Philox4x32-10
 *   with key = seed and subsequence = site (src/random.cu:15-35), one draw per
 *   site per half-sweep (src/device_2d.cu:96-97).
 * SA_RNG_MT19937_64: the CPU reference's stream, one std::mt19937_64 per system
 *   (src/cpu_2dp.hpp:35-36, src/cpu_3d.hpp:37-39) generated on the device and
 *   consumed as cpu_2d / cpu_2dp / cpu_3d consume it: set_seed reseeds it
 *   (src/cpu_3d.cpp:210), init_J takes dim*N outputs (src/cpu_2dp.cpp:243-260,
 *   src/cpu_3d.cpp:281-301), init_rand N (src/cpu_3d.cpp:257-263), and a sweep
 *   one uniform_real_distribution<double> draw per site in the reference's
 *   visiting order (src/cpu_3d.cpp:94-105, :130). Spins, couplings and
 *   energies then match the unmodified reference CPU classes bit for bit.
 *   Switching to it reseeds the generator with the current seed. */
int sa_sys_set_rng_mode(sa_system_t sys, int mode);
int sa_sys_get_rng_mode(sa_system_t sys, int* mode);
/* The colour of each sweep's first half-sweep (default 0). The reference's
 * GPU systems hold two lattices and update one from the other
 * (src/gpu_2d.cu:109-120): of the two configurations they carry, the second
 * updates its colour-1 sites first (draw t+2n) and its colour-0 sites second
 * (t+2n+1). Colour 1 gives that order; such a system also draws its initial
 * spins from a counter range of its own. Philox mode only. */
int sa_sys_set_first_colour(sa_system_t sys, int colour);
int sa_sys_get_first_colour(sa_system_t sys, int* colour);
/* The reference's SPLIT_H update (src/device_2d.cu:27-50,
 * src/device_3d.cu:216-245, tables src/gpu_2d.cu:133-139,
 * src/gpu_3d.cu:57-63), off by default as in the reference's build: a flip is
 * accepted in two parts, each site drawing two uniforms per half-sweep (draw
 * t+2m for the bonds, t+2m+1 for the field). The bond part for n satisfied of
 * z bonds is accepted always when 2n <= z, else iff u1 < float(exp(-2j/T)),
 * j = 2n - z (open-x border sites count their forced bond: j = 2n - 5); an up
 * spin's field part iff u2 < float(exp(-2h/T)) (not clamped), a down spin's
 * always. In 3D a site with a coordinate 0 or L-1 uses its field draw for the
 * bond part too, as the reference's boundary branch does. Philox mode only;
 * sweeps run two launches per sweep. */
int sa_sys_set_split_field(sa_system_t sys, int on);
int sa_sys_get_split_field(sa_system_t sys, int* on);
/* The reference CPU classes' own checkpoint record, byte for byte as
 * cpu_2dp::save / cpu_3d::save write it (src/cpu_2dp.cpp:444-456,
 * src/cpu_3d.cpp:449-461): L, T, h, spins, the reference-layout couplings and
 * the std::mt19937_64 state. Saving needs SA_RNG_MT19937_64 mode (the record
 * carries that generator); loading switches the system to it, so a run can
 * move between the reference's CPU binary and this engine mid-stream.
 * buf == NULL: *len receives the size. */
int sa_sys_save_reference(sa_system_t sys, void* buf, size_t cap, size_t* len);
int sa_sys_load_reference(sa_system_t sys, const void* buf, size_t len);
/* RNG position (for checkpoints): draw counter and spin-init epoch. */
int sa_sys_get_rng(sa_system_t sys, uint64_t* seed, uint64_t* draw, uint64_t* epoch);
int sa_sys_set_rng(sa_system_t sys, uint64_t seed, uint64_t draw, uint64_t epoch);
/* Wait for the system's queued work. */
int sa_sys_sync(sa_system_t sys);
/* save()/load() replacement (src/gpu_2d.cu:327-412): a self-describing
 * checkpoint (lattice, L, T, h, seed, draw, epoch, spins, own couplings).
 * sa_sys_save with buf==NULL reports the size in *len. */
int sa_sys_save(sa_system_t sys, void* buf, size_t cap, size_t* len);
int sa_sys_load(sa_system_t sys, const void* buf, size_t len);

/* The exchange schedule of parallel_tempering<> for n temperatures
 * (src/parallel_tempering.hpp:28-30, :59, :112-114): std::mt19937(123)
 * driving uniform_int_distribution<int>(0, n-2) then
 * uniform_real_distribution<double>; entries skip .. skip+count-1 into pair[]
 * and r[] (host). */
int sa_pt_sequence(int n, long skip, long count, int32_t* pair, double* r);

/* The same generator as an object that keeps its position, for drivers that
 * draw one attempt at a time and for checkpoints: the members gen, uni_int
 * and uni_double of parallel_tempering<> (src/parallel_tempering.hpp:28-30),
 * created as its constructor creates them (:59) for n temperatures. */
typedef struct sa_pt_gen* sa_pt_gen_t;
int sa_pt_gen_create(int n, sa_pt_gen_t* out);
int sa_pt_gen_destroy(sa_pt_gen_t g);
/* The next `count` attempts (src/parallel_tempering.hpp:112-114): pair[k] =
 * uni_int(gen), then r[k] = uni_double(gen). */
int sa_pt_gen_next(sa_pt_gen_t g, long count, int32_t* pair, double* r);
/* update_T's widening of the pair range by one (src/parallel_tempering.hpp:
 * 410): uni_int becomes uniform_int_distribution<int>(a, b+1). */
int sa_pt_gen_widen(sa_pt_gen_t g);
/* The three objects' bytes as parallel_tempering<>::save writes them, in its
 * order gen, uni_int, uni_double (src/parallel_tempering.hpp:284-287; the
 * raw libstdc++ objects, 5024 bytes on LP64); load takes the same bytes
 * (:324-327). buf == NULL: *len receives the size. */
int sa_pt_gen_save(sa_pt_gen_t g, void* buf, size_t cap, size_t* len);
int sa_pt_gen_load(sa_pt_gen_t g, const void* buf, size_t len);
/* The reference's exchange mask for one pair (src/parallel_tempering.hpp:
 * 141-162): bit j iff dE*dB > 0 || r < exp(dB*dE), dE = -(Ei[j]-Ej[j]) (float),
 * dB = 1/Ti - 1/Tj. Host-only arithmetic. */
uint64_t sa_pt_mask(const float* Ei, const float* Ej, double Ti, double Tj, double r);

/* annealing<gpu_sys> on the device (src/annealing.hpp:67-100) for one system:
 * nsteps steps, step k at temperature T[k] with `sweeps` sweeps, measuring
 * after every sweep i (inside the step) with i % stride == 0 (stride 0: never)
 * and keeping the running maximum of the float -H = E + h*M per replica
 * (the reference's min_E) in min_E[64] (host). step_E (host, nsteps*64, may
 * be NULL) receives the integer E of the last measurement of every step.
 * The reference's geometric cooling T *= alfa is the schedule T[k] =
 * T0*alfa^k. Leaves the system at temperature T[nsteps-1]. Synchronous. */
int sa_sys_anneal(sa_system_t sys, const double* T, int nsteps, int sweeps, int stride, float* min_E,
                  int64_t* step_E);

/* Allocation-free energy measurement (no counterpart in the reference; the
 * reference measures through its system object, which owns its buffers).
 * Same result as sa_sys_measure -- E[j], M[j] per replica bit j -- for a
 * lattice whose spins and own couplings the caller already holds on the
 * device in the internal layout (see sa_sys_device_buffers), written to the
 * caller's DEVICE arrays d_E[64], d_M[64], asynchronously on `stream`.
 * For callers that cannot allocate device memory when they need an energy
 * (a process that reserved its HBM budget up front, or a loop that cannot
 * afford cudaMalloc's latency and implicit synchronisation): it calls no
 * allocator. Its scratch is a fixed 256 KB array in the library's device
 * image (512 partials of 128 counters), present on every device that loads
 * the library until the process exits; lattices above 67,108,864 sites are
 * rejected with SA_ERR_BUDGET. The first call on a device looks up the
 * array's device address, so make that first call before any stream
 * capture. All calls share the array: calls that overlap on the GPU (e.g. on
 * two streams) race and must be ordered by the caller. */
int sa_measure_noalloc(int lattice, int L, const uint64_t* d_spins, const uint64_t* d_J,
                       int64_t* d_E, int64_t* d_M, void* stream);

/* Device pointers of the internal layout (read-only use by advanced callers):
 * spins [colour][row][k] and own couplings [axis][colour][row][k]. */
int sa_sys_device_buffers(sa_system_t sys, uint64_t** d_spins, uint64_t** d_J);

#ifdef __cplusplus
}
#endif
#endif /* SA_B200_H */
