// One "pass" of the B200 FFT provider: a batch of line FFTs executed by a single
// kernel launch, with everything a pass needs fused into its load and store.
//
// A pass sees its data as lines. Line (o, c) has elements k = 0..n-1 at
//   addr = (o / d) * hi + (o % d) * lo + c * cs + k * ks          (in complex units)
// separately for the input and the output layout. A CTA owns one tile: a fixed
// outer index o and `w` consecutive columns c. The FFT along k is a Stockham
// autosort sequence of radix-R stages held in registers, exchanging through
// shared memory between stages.
//
// Fused extras (all optional):
//   load : zero padding (element index g >= in_len reads 0), pre-multiply by a table
//          indexed by g, conjugation (inverse transforms run as conj-FFT-conj);
//   mid  : point-wise multiply by a table, conjugation, and a second FFT (Bluestein
//          convolution in one kernel);
//   store: conjugation, the four-step twiddle W_N^(sign*k*sel), post-multiply by a
//          table indexed by g, the normalization scale, truncation (g >= out_len is
//          not written).
// The element index is g = k * g_k + sel with sel = 0, c, (o % sel_d) or (c % sel_d).
//
// This header is plain C++ so host planning code and device code share it.
#pragma once

#include <cstdint>

namespace sfb {

constexpr int kMaxStages = 16;

enum : int { kModeK = 0, kModeC = 1 };         // thread mapping / coalesced dimension
enum : int { kSelNone = 0, kSelCol = 1, kSelOuterLo = 2, kSelColMod = 3 };

struct LineLayout {
    int64_t hi = 0, lo = 0, d = 1, cs = 0, ks = 1;
};

struct StageSeq {
    int nstages = 0;
    int radix[kMaxStages] = {};
    int ns[kMaxStages] = {};      // product of the radices before this stage
    int tw_off[kMaxStages] = {};  // offset of this stage's twiddles in `tw` (complex units)
    const void* tw = nullptr;     // per stage: [ns][radix-1] of exp(-2 pi i r j / (ns*radix))
};

struct PassParams {
    int n = 1;           // FFT length along k
    int tpl = 1;         // threads per line
    int w = 1;           // lines (columns) per CTA tile
    int mode = kModeK;   // kModeK: threads walk k; kModeC: threads walk columns
    int pitch = 0;       // shared-memory line pitch (kModeK) in complex units
    int pad_shift = 31;  // shared-memory padding: one element per 2^pad_shift
    int64_t n_outer = 1, n_cols = 1, col_tiles = 1, tiles = 1;
    LineLayout in, out;

    // element index g = k * g_k + sel
    int64_t g_k = 1;
    int sel_mode = kSelNone;
    int64_t sel_d = 1;
    int64_t in_len = 0;   // input elements with g >= in_len read as zero
    int64_t out_len = 0;  // outputs with g >= out_len are not stored

    const void* premul = nullptr;     // [in_len] multiplied on load (indexed by g)
    int conj_in = 0;
    StageSeq fft1;
    const void* pointwise = nullptr;  // multiplied after fft1, indexed k + sel * pw_stride
    int64_t pw_stride = 0;
    int conj_mid = 0;
    StageSeq fft2;                    // nstages == 0: no second FFT
    int conj_out = 0;
    const void* tw4_hi = nullptr;     // four-step twiddle W^(m) = hi[m >> shift] * lo[m & mask]
    const void* tw4_lo = nullptr;
    int tw4_shift = 0;
    int tw4_sign = 0;                 // 0: off; -1 / +1: exponent sign
    const void* postmul = nullptr;    // indexed by g on store
    double scale = 1.0;
    int store_via_smem = 0;           // transpose through shared memory before storing
    // Direction override of a whole plan (conj(F(conj x))): conjugate the raw input before
    // the pre-multiply and the final value after the post-multiply and scale. Used instead of
    // conj_in / conj_out by passes that carry premul / postmul tables (Bluestein), where the
    // plan's own conjugations sit between the FFTs and the chirp products.
    int flip_in = 0, flip_out = 0;
    // Rader passes: int32 permutations of the line (load element g from perm_in[g], store
    // element g to perm_out[g], both relative to the line start)
    const void* perm_in = nullptr;
    const void* perm_out = nullptr;
    // Size-specialised four-step row pass: row l (= o*ts_rows + k1) stored at
    // (l / ts_rows) * ts_line + l % ts_rows + k * ts_rows.
    int64_t ts_rows = 0, ts_line = 0;
};

}  // namespace sfb
