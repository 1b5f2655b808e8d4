// Host-side planner of the B200 FFT provider.
//
// Turns (shape, batch, precision, direction, normalization) into a list of
// fused passes (pass_params.h) plus FP64 tables. It has no CUDA dependency:
// the provider uploads the tables (cast to the plan precision) and binds the
// device pointers; tests drive the same plans through a CPU emulator.
//
// Decomposition rules (per axis of length L, processed last axis first):
//   * L == 1                         -> no pass (a copy pass if every axis is 1);
//   * 7-smooth and fits one CTA      -> one pass (Stockham, shared memory);
//   * 7-smooth and larger            -> four-step: L = N1 * N2, column pass with the
//                                       W_L^(n2*k1) twiddle fused into its store, then a
//                                       row pass storing transposed (two passes);
//   * prime, L-1 in the catalog      -> Rader: a cyclic convolution of length M = L-1
//     (contiguous axis)                 over the permuted line (generator powers), one fused
//                                       pass or three passes as below;
//   * otherwise (Bluestein)          -> convolution of length M (the smallest 7-smooth
//                                       M >= 2L-2): one fused pass when M fits a CTA,
//                                       else three passes over an M-padded scratch.
// The normalization scale is fused into the store of the last pass.
#pragma once

#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "pass_params.h"

namespace sfb {

enum class Buf : int { Input = 0, Output = 1, Scratch = 2 };

struct TableIds {
    int tw1 = -1, tw2 = -1, premul = -1, pointwise = -1, postmul = -1, tw4_hi = -1, tw4_lo = -1;
    int tc_tw = -1;  // two-level W_N^k table of the tensor-core kernel
    int cl_base = -1;  // base twiddles of the pipelined cluster kernel's 256-point FFTs
    int perm_in = -1, perm_out = -1;  // Rader permutations (PlanSpec::index_tables)
};

struct KernelChoice {
    int maxv = 16;   // register capacity (complex values per thread per stage)
    int maxt = 256;  // __launch_bounds__ of the instantiation
};

struct PassSpec {
    PassParams p;
    TableIds tables;
    Buf src = Buf::Input, dst = Buf::Output;
    KernelChoice kc;
    int threads = 0;         // blockDim.x
    int64_t smem_bytes = 0;  // dynamic shared memory
    std::string kind;        // "single", "fourstep_cols", "fourstep_rows", "bluestein_fused", ...
    int axis = 0;
    int64_t bytes_moved = 0; // HBM bytes this pass reads + writes (data, not tables)
    int fixed_id = -1;       // size-specialised kernel (fixed_catalog.h), -1 = generic kernel
    int fixed_feat = 0;      // its feature (kFixedPlain / kFixedTw4 / kFixedTStore)
    bool tw_base = false;    // tables.tw1 holds base twiddles W_(ns*R)^jm (size-specialised kernels)
    // Which line count is proportional to the plan's batch: 0 = n_outer, 1 = n_cols
    // (lets a plan for up to B transforms run the first b <= B).
    int batch_dim = 1;
    int cluster_id = -1;     // cluster kernel (cluster_catalog.h) for a whole long line
    int piped_id = -1;       // copy-engine-pipelined kernel (piped_catalog.h), used when the
                             // buffers are 16-byte aligned; otherwise fixed_id runs
    int cl_n1 = 0, cl_n2 = 0, cl_p = 0;
    int tc_id = -1;          // split-precision tensor-core kernel (tc_catalog.h), float plans only
    bool tma = false;        // four-step column pass with a TMA-staged variant of fixed_id (tma_cols_kernel.cuh)
    int blue_id = -1;        // size-specialised Bluestein kernel (bluestein_catalog.h)
    int blue_kind = -1;      // its kind: kBlueFused / kBlueColsFwd / kBlueRowsConv / kBlueColsInv
    bool cluster_pipe = false;  // cluster pass on the pipelined 16-CTA kernel (cluster_pipe.cu)
    // Rader pass (blue_id then names the catalog kernel whose Rader instantiation runs):
    // gather / scatter through the permutation tables; rader_dc: the convolution pass that
    // also stores X[0], reading x[0] from the axis input rader_src
    bool rader = false;
    bool rader_dc = false;
    Buf rader_src = Buf::Input;
    // runtime-length pass on the contiguous-layout kernel (lean_kernel.cuh) instead of the
    // general one; lean_feat: kLeanPlain / kLeanTw4. A lean pass reads base twiddles
    // (tw_base), so it only runs on the lean kernel.
    bool lean = false;
    int lean_feat = 0;
};

// The lean kernel's instantiations (lean_variants.cu): float with 16 values per thread, double
// with 8 (or 16 up to 512 threads); CTA bounds 256 / 512 / 1024.
inline bool lean_variant_exists(bool dbl, int maxv, int maxt) {
    if (maxt != 256 && maxt != 512 && maxt != 1024) return false;
    if (!dbl) return maxv == 16;
    return maxv == 8 || (maxv == 16 && maxt <= 512);
}

// One entry of cluster_catalog.h as seen by the host.
struct ClusterEntry {
    int id, dbl, n1, n2, p, tpl1, tpl2, maxt, minb;
    int r1[kMaxStages], r2[kMaxStages];
    int ns1, ns2;
};
// Entries for a line length; `prefer_p` (0 = catalog order) picks the cluster size.
const ClusterEntry* find_cluster(bool dbl, int64_t n, int prefer_p);

// One entry of fixed_catalog.h as seen by the host.
enum : int { kFixedPlain = 0, kFixedTw4 = 1, kFixedTStore = 2 };
struct FixedEntry {
    int id, dbl, modec, feat, n, tpl, w, maxt;
    int radices[kMaxStages];
    int nstages;
};
const FixedEntry* find_fixed(bool dbl, int mode, int n, int feat);
// A fused four-step kernel (fused4_catalog.h) runs these column and row entries together.
bool has_fused4(bool dbl, int col_id, int row_id);

// One entry of piped_catalog.h as seen by the host.
struct PipedEntry {
    int id, dbl, n, tpl, maxt;
    int radices[kMaxStages];
    int nstages;
};
const PipedEntry* find_piped(bool dbl, int n);

// One entry of bluestein_catalog.h as seen by the host.
enum : int { kBlueFused = 0, kBlueColsFwd = 1, kBlueRowsConv = 2, kBlueColsInv = 3 };
struct BlueEntry {
    int id, dbl, kind, n, tpl, w, maxt;
    int radices[kMaxStages];
    int nstages;
};
const BlueEntry* blue_entries(int* count);

// One entry of tc_catalog.h (split-precision tensor-core kernels, complex<float> only).
struct TcEntry {
    int id, r, s, l, cols;
    int n, threads;
    int64_t smem;
};
// Entry for a line length and layout (cols: the lines are adjacent columns), or nullptr.
const TcEntry* find_tc(int n, bool cols);

struct PlanRequest {
    bool dbl = false;
    int direction = -1;      // -1 forward, +1 backward
    int normalization = 0;   // 0 none, 1 forward, 2 backward, 3 orthogonal
    bool in_place = false;
    std::vector<uint64_t> shape;
    uint64_t batch = 1;
    // tuning knobs (0 = heuristic)
    int force_maxv = 0;
    int force_w = 0;
    int force_n1 = 0;        // four-step column length (0: the most balanced split)
    int smem_limit = 0;      // bytes, 0 = device default (227 KB)
    bool no_fixed = false;   // force the generic kernel (tests, tuning)
    bool no_cluster = false; // force the two-pass four-step for long lines
    bool no_piped = false;   // never use the copy-engine-pipelined kernels
    // Lines that fit one block but have a fused four-step kernel (fused4_catalog.h) run as a
    // four-step through it (column and row passes in one launch, L2-resident intermediate)
    // instead of the single pass; needs at least 3 lines.
    bool fused_single = false;
    bool use_tma = false;    // four-step column passes on the TMA-staged kernels (opt-in: measured
                             // level with the plain size-specialised kernel on B200)
    int cluster_p = 0;       // > 0: put long lines on the cluster kernel of this cluster size
    bool device_spectrum = false;  // leave Bluestein chirp/spectrum tables to the device (zeroed here)
    // complex<float> only: run the radix-16 butterflies of eligible single-pass axes as BF16
    // hi/lo matrix products on the tensor cores (FP32 accumulation); other passes stay FP32
    bool split_bf16 = false;
    // bit ax set: axis ax is an index of the batch, not transformed (interleaved-batch layouts:
    // transforms down the columns of a dense array run as the other axes' passes alone)
    uint32_t skip_axes = 0;
    // complex<double> 65536-point lines: the cluster pass (cluster_p = 16) on the pipelined
    // cluster kernel (opt-in)
    bool cluster_pipe = false;
    // prime lengths L take Bluestein's convolution even where the catalog covers L - 1 (Rader)
    bool no_rader = false;
};

// A Bluestein axis whose chirp and chirp spectrum the provider generates on the device
// (PlanRequest::device_spectrum): chirp[n] = conj(h_n), h_n = exp(-i*sgn*pi*(n^2 mod 2L)/L),
// spectrum = FFT_M(h zero-padded, mirrored) / M, permuted K'[k1*n2+k2] = K[k1+n1*k2] when large.
struct BluesteinJob {
    int64_t L = 0, M = 0, n1 = 0, n2 = 0;
    int sgn = -1;
    bool large = false;
    int chirp_table = -1, spectrum_table = -1;
};

struct PlanSpec {
    PlanRequest req;
    std::vector<BluesteinJob> bluestein_jobs;
    std::string tuning;  // autotuner report (JSON object), empty when not tuned
    uint64_t elements = 0, transform_size = 0;
    double scale = 1.0;
    std::vector<std::vector<std::complex<double>>> tables;
    // Entries of each table; a table whose data is empty but whose size is not is generated on
    // the device (Bluestein chirp and spectrum with PlanRequest::device_spectrum).
    std::vector<size_t> table_sizes;
    std::vector<std::vector<int32_t>> index_tables;  // int32 tables (Rader permutations)
    std::vector<PassSpec> passes;
    uint64_t scratch_elements = 0;
};

// Throws std::invalid_argument / std::runtime_error with a message on failure.
PlanSpec make_plan(const PlanRequest& req);

// Element count with the reference's validation (rank 1..3, non-zero sizes, overflow).
uint64_t checked_element_count(const std::vector<uint64_t>& shape, uint64_t batch);
// Normalization scale as the reference computes it (in double).
double normalization_scale(int mode, int direction, uint64_t transform_size);

// Helpers exposed for tests.
bool smooth7(uint64_t n);
uint64_t bluestein_length(uint64_t len);
bool is_prime(uint64_t n);
uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t m);
uint64_t primitive_root(uint64_t p);  // p prime
std::vector<int> choose_radices(int n, int maxv);
int threads_per_line(int n, const std::vector<int>& radices, int maxv);
std::string describe_plan(const PlanSpec& plan);  // JSON

// exp(-2 pi i num / den), with exact argument reduction (num reduced mod den, octant symmetry).
std::complex<double> cis_neg(int64_t num, int64_t den);

// Reference-quality FP64 FFT on the host (Stockham, same radices as the device).
void host_fft_fp64(std::vector<std::complex<double>>& a, int sign);

}  // namespace sfb
