#include "planner.hpp"

#include "cluster_catalog.h"
#include "fixed_catalog.h"
#include "fused4_catalog.h"
#include "piped_catalog.h"
#include "tc_catalog.h"
#include "bluestein_catalog.h"
#include "tc_shape.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>

namespace sfb {

namespace {

constexpr int kSmemDefault = 227 * 1024;
constexpr int64_t kNoLimit = std::numeric_limits<int64_t>::max() / 4;

struct Factors {
    int e2 = 0, e3 = 0, e5 = 0, e7 = 0;
};

bool factor7(uint64_t n, Factors& f) {
    if (n == 0) return false;
    while (n % 2 == 0) { n /= 2; ++f.e2; }
    while (n % 3 == 0) { n /= 3; ++f.e3; }
    while (n % 5 == 0) { n /= 5; ++f.e5; }
    while (n % 7 == 0) { n /= 7; ++f.e7; }
    return n == 1;
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

int pad_shift_for(bool dbl) { return dbl ? 3 : 4; }

int kmode_pitch(int n, int pad_shift) {
    int p = n + (n >> pad_shift);
    if ((p & 1) == 0) p += 1;  // odd pitch: columns of the tile fall in distinct banks
    return p;
}

struct SingleCfg {
    bool ok = false;
    KernelChoice kc;
    std::vector<int> radices;
    int tpl = 0;
};

// Largest CTA the kernel variant may use, given the register arrays it holds.
int max_threads_for(bool dbl, int maxv) {
    if (dbl && maxv >= 16) return 512;
    return 1024;
}

SingleCfg single_cfg(int64_t n, bool dbl, int force_maxv) {
    SingleCfg best;
    if (n <= 0 || n > (1 << 20) || !smooth7(static_cast<uint64_t>(n))) return best;
    std::vector<int> cands;
    if (force_maxv) cands = {force_maxv};
    else if (dbl) cands = {8, 16};
    else cands = {16};
    for (int maxv : cands) {
        auto r = choose_radices(static_cast<int>(n), maxv);
        const int tpl = threads_per_line(static_cast<int>(n), r, maxv);
        if (tpl > max_threads_for(dbl, maxv)) continue;
        best.ok = true;
        best.kc.maxv = maxv;
        best.radices = r;
        best.tpl = tpl;
        return best;
    }
    return best;
}

int maxt_for(int threads) {
    if (threads <= 256) return 256;
    if (threads <= 512) return 512;
    return 1024;
}

// Process-wide cache of generated tables: stage twiddles and four-step twiddles depend only
// on their radix sequence / length, so plans of the same lengths reuse them.
std::mutex g_table_mu;
std::map<std::vector<int64_t>, std::shared_ptr<const std::vector<std::complex<double>>>> g_tables;

template <class Make>
std::shared_ptr<const std::vector<std::complex<double>>> cached_table(std::vector<int64_t> key, Make make) {
    {
        std::lock_guard<std::mutex> lock(g_table_mu);
        auto it = g_tables.find(key);
        if (it != g_tables.end()) return it->second;
    }
    auto t = std::make_shared<const std::vector<std::complex<double>>>(make());
    std::lock_guard<std::mutex> lock(g_table_mu);
    if (g_tables.size() > 4096) g_tables.clear();  // bound the cache
    g_tables[key] = t;
    return t;
}

struct Builder {
    PlanSpec& plan;
    const PlanRequest& req;
    int cs;
    int smem_limit;
    std::map<std::vector<int>, int> seq_tables;  // radix sequence -> twiddle table id

    int add_table(std::vector<std::complex<double>> t) {
        plan.table_sizes.push_back(t.size());
        plan.tables.push_back(std::move(t));
        return static_cast<int>(plan.tables.size()) - 1;
    }

    int add_index_table(std::vector<int32_t> t) {
        plan.index_tables.push_back(std::move(t));
        return static_cast<int>(plan.index_tables.size()) - 1;
    }

    // A table of n entries the device fills (no host data).
    int add_device_table(size_t n) {
        plan.table_sizes.push_back(n);
        plan.tables.emplace_back();
        return static_cast<int>(plan.tables.size()) - 1;
    }

    // Stockham stage sequence for length n with the given radices; twiddle table shared per (n, radices).
    StageSeq make_seq(int n, const std::vector<int>& radices, int maxv, int* table_id) {
        StageSeq s;
        if (static_cast<int>(radices.size()) > kMaxStages) throw std::runtime_error("too many FFT stages");
        s.nstages = static_cast<int>(radices.size());
        int ns = 1, off = 0;
        for (int i = 0; i < s.nstages; ++i) {
            s.radix[i] = radices[i];
            s.ns[i] = ns;
            s.tw_off[i] = off;
            off += ns * (radices[i] - 1);
            ns *= radices[i];
        }
        if (ns != n) throw std::runtime_error("radix product mismatch");
        (void)maxv;
        const std::vector<int>& key = radices;
        auto it = seq_tables.find(key);
        if (it != seq_tables.end()) {
            *table_id = it->second;
            return s;
        }
        std::vector<int64_t> ckey(radices.begin(), radices.end());
        ckey.push_back(-100);
        const StageSeq sc = s;
        auto tw = cached_table(ckey, [&] {
            std::vector<std::complex<double>> t(std::max(off, 1));
            int ns2 = 1;
            for (int i = 0; i < sc.nstages; ++i) {
                const int R = radices[i];
                for (int jm = 0; jm < ns2; ++jm)
                    for (int r = 1; r < R; ++r)
                        t[sc.tw_off[i] + jm * (R - 1) + (r - 1)] =
                            cis_neg(static_cast<int64_t>(r) * jm, static_cast<int64_t>(ns2) * R);
                ns2 *= R;
            }
            return t;
        });
        *table_id = add_table(*tw);
        seq_tables[key] = *table_id;
        return s;
    }

    // Base-twiddle table of the size-specialised kernels: for each stage, W_(ns*R)^jm, jm < ns.
    int base_table(const std::vector<int>& radices) {
        std::vector<int> key = radices;
        key.push_back(-1);  // distinct from the full-table key
        auto it = seq_tables.find(key);
        if (it != seq_tables.end()) return it->second;
        std::vector<int64_t> ckey(radices.begin(), radices.end());
        ckey.push_back(-200);
        auto tw = cached_table(ckey, [&] {
            std::vector<std::complex<double>> t;
            int64_t ns = 1;
            for (int R : radices) {
                for (int64_t jm = 0; jm < ns; ++jm) t.push_back(cis_neg(jm, ns * R));
                ns *= R;
            }
            if (t.empty()) t.push_back(1.0);
            return t;
        });
        const int id = add_table(*tw);
        seq_tables[key] = id;
        return id;
    }

    // Split-precision tensor-core kernel for a plain single-pass axis of a float plan: the
    // line length must be a catalog length (radix-16 powers) and the pass must carry no
    // fused extras (those are the Bluestein and four-step passes, which stay FP32).
    void try_tc(PassSpec& ps) {
        PassParams& p = ps.p;
        if (req.dbl || ps.kind != "single" || p.fft2.nstages != 0 || p.in_len != p.n || p.out_len != p.n ||
            ps.tables.premul >= 0 || ps.tables.pointwise >= 0 || ps.tables.postmul >= 0 || p.tw4_sign != 0 ||
            p.store_via_smem || p.ts_rows)
            return;
        const bool cols = p.mode == kModeC;
        const TcEntry* e = find_tc(p.n, cols);
        if (!e || e->smem > smem_limit) return;
        if (cols ? (p.in.cs != 1 || p.out.cs != 1) : (p.in.ks != 1 || p.out.ks != 1)) return;
        const int64_t n = p.n;
        auto tw = cached_table({n, -400}, [&] {
            // two levels: W_n^(64a) for a < ceil(n/64), then W_n^b for b < 64
            std::vector<std::complex<double>> t;
            for (int64_t a = 0; a < (n + 63) / 64; ++a) t.push_back(cis_neg(64 * a, n));
            for (int64_t b = 0; b < 64; ++b) t.push_back(cis_neg(b, n));
            return t;
        });
        ps.tables.tc_tw = add_table(*tw);
        ps.tc_id = e->id;
        ps.threads = e->threads;
        ps.smem_bytes = e->smem;
        p.w = e->l;
        p.col_tiles = (p.n_cols + p.w - 1) / p.w;
        p.tiles = p.n_outer * p.col_tiles;
    }

    void use_base_table(PassSpec& ps) {
        std::vector<int> r(ps.p.fft1.radix, ps.p.fft1.radix + ps.p.fft1.nstages);
        ps.tables.tw1 = base_table(r);
        ps.tw_base = true;
    }

    void add_tw4(PassSpec& ps, int64_t ntot, int sign) {
        int shift = 0;
        while ((int64_t(1) << (2 * shift)) < ntot) ++shift;  // 2^shift >= sqrt(ntot)
        const int64_t B = int64_t(1) << shift;
        const int64_t nhi = (ntot + B - 1) / B + 1;
        auto hi = cached_table({ntot, B, -300}, [&] {
            std::vector<std::complex<double>> t(nhi);
            for (int64_t q = 0; q < nhi; ++q) t[q] = cis_neg(q * B, ntot);
            return t;
        });
        auto lo = cached_table({ntot, B, -400}, [&] {
            std::vector<std::complex<double>> t(B);
            for (int64_t r = 0; r < B; ++r) t[r] = cis_neg(r, ntot);
            return t;
        });
        ps.tables.tw4_hi = add_table(*hi);
        ps.tables.tw4_lo = add_table(*lo);
        ps.p.tw4_shift = shift;
        ps.p.tw4_sign = sign;
    }

    // Fill launch geometry for a pass whose FFT length is p.n and mode is set.
    // Lines per CTA of a runtime-parameterised four-step pass: about 256 threads (several CTAs
    // per SM; CTAs of ~1000 threads leave one per SM, every stage barrier then stalls the SM),
    // at least 4 lines (32-byte segments) and at most `cap`, a power of two.
    static int fourstep_w(int tpl, int cap) {
        int w = std::max(4, std::min(cap, 256 / std::max(1, tpl)));
        while (w & (w - 1)) w &= w - 1;
        return w;
    }

    void geometry(PassSpec& ps, const SingleCfg& cfg, int want_w) {
        PassParams& p = ps.p;
        p.tpl = cfg.tpl;
        ps.kc = cfg.kc;
        const int max_threads = max_threads_for(req.dbl, cfg.kc.maxv);
        int w;
        if (p.mode == kModeK) {
            p.pad_shift = pad_shift_for(req.dbl);
            p.pitch = kmode_pitch(p.n, p.pad_shift);
            // lines per CTA: about 256 threads, a power of two (the lean kernel's tiles)
            w = want_w > 0 ? want_w : std::max(1, 256 / cfg.tpl);
            if (want_w <= 0)
                while (w & (w - 1)) w &= w - 1;
            w = static_cast<int>(std::min<int64_t>(w, p.n_cols));
            while (w > 1 && (w * cfg.tpl > max_threads ||
                             static_cast<int64_t>(w) * p.pitch * cs > smem_limit))
                --w;
            ps.smem_bytes = static_cast<int64_t>(w) * p.pitch * cs;
        } else {
            w = want_w > 0 ? want_w : (req.dbl ? 8 : 16);
            w = static_cast<int>(std::min<int64_t>(w, p.n_cols));
            while (w > 1 && (w * cfg.tpl > max_threads ||
                             static_cast<int64_t>(w) * p.n * cs > smem_limit))
                --w;
            ps.smem_bytes = static_cast<int64_t>(w) * p.n * cs;
        }
        p.w = std::max(w, 1);
        ps.threads = round_up(p.w * cfg.tpl, 32);
        if (ps.threads > max_threads) throw std::runtime_error("FFT pass needs too many threads per CTA");
        if (ps.smem_bytes > smem_limit) throw std::runtime_error("FFT pass exceeds shared memory");
        ps.kc.maxt = maxt_for(ps.threads);
        p.col_tiles = (p.n_cols + p.w - 1) / p.w;
        p.tiles = p.n_outer * p.col_tiles;
    }

    // Switch a plain single pass to its size-specialised kernel when the catalog has one.
    void try_fixed(PassSpec& ps, const SingleCfg& cfg) {
        if (req.no_fixed || (req.force_maxv && req.force_maxv != cfg.kc.maxv)) return;
        PassParams& p = ps.p;
        const FixedEntry* e = find_fixed(req.dbl, p.mode, p.n, kFixedPlain);
        if (!e) return;
        // The entry's own radix sequence (it may use butterflies the runtime-parameterised
        // kernel does not have, such as the prime-factor radix 15).
        if (e->nstages != p.fft1.nstages || !std::equal(e->radices, e->radices + e->nstages, p.fft1.radix)) {
            StageSeq q;
            q.nstages = e->nstages;
            int ns = 1;
            for (int i = 0; i < e->nstages; ++i) {
                q.radix[i] = e->radices[i];
                q.ns[i] = ns;
                ns *= e->radices[i];
            }
            p.fft1 = q;
        }
        if (p.mode == kModeK) {
            if (p.in.ks != 1 || p.out.ks != 1 || p.n_outer != 1) return;
            int w = req.force_w > 0 ? req.force_w : std::max(1, 256 / e->tpl);
            w = static_cast<int>(std::min<int64_t>(w, p.n_cols));
            while (w > 1 && (w * e->tpl > e->maxt || static_cast<int64_t>(w) * p.pitch * cs > smem_limit)) --w;
            p.w = w;
            ps.threads = round_up(w * e->tpl, 32);
            ps.smem_bytes = static_cast<int64_t>(w) * p.pitch * cs;
        } else {
            if (p.in.cs != 1 || p.out.cs != 1 || p.in.d != 1 || p.out.d != 1) return;
            p.w = e->w;
            ps.threads = round_up(e->w * e->tpl, 32);
            ps.smem_bytes = static_cast<int64_t>(e->w) * p.n * cs;
            if (ps.smem_bytes > smem_limit) return;
        }
        if (ps.threads > e->maxt) return;
        p.tpl = e->tpl;
        p.col_tiles = (p.n_cols + p.w - 1) / p.w;
        p.tiles = p.n_outer * p.col_tiles;
        ps.kc.maxt = e->maxt;
        ps.fixed_id = e->id;
        ps.fixed_feat = kFixedPlain;
        use_base_table(ps);
        if (p.mode == kModeK && !req.no_piped && (p.in.cs * cs) % 16 == 0 && (p.out.cs * cs) % 16 == 0) {
            if (const PipedEntry* pe = find_piped(req.dbl, p.n)) {
                bool same = pe->nstages == p.fft1.nstages;
                for (int i = 0; same && i < pe->nstages; ++i) same = pe->radices[i] == p.fft1.radix[i];
                if (same) ps.piped_id = pe->id;
            }
        }
    }

    // Four-step passes of a contiguous axis on their size-specialised kernels.
    void try_fixed_fourstep(PassSpec& ps, int feat, int64_t rows = 0, int64_t line = 0) {
        if (req.no_fixed) return;
        PassParams& p = ps.p;
        const FixedEntry* e = find_fixed(req.dbl, p.mode, p.n, feat);
        if (!e) return;
        // the entry's own radix sequence (it may use butterflies the runtime-parameterised
        // kernel does not have, such as the prime-factor radix 15)
        if (e->nstages != p.fft1.nstages || !std::equal(e->radices, e->radices + e->nstages, p.fft1.radix)) {
            StageSeq q;
            q.nstages = e->nstages;
            int ns = 1;
            for (int i = 0; i < e->nstages; ++i) {
                q.radix[i] = e->radices[i];
                q.ns[i] = ns;
                ns *= e->radices[i];
            }
            if (ns != p.n) return;
            p.fft1 = q;
        }
        const int threads = round_up(e->w * e->tpl, 32);
        if (threads > e->maxt) return;
        if (feat == kFixedTw4) {
            const int64_t smem = static_cast<int64_t>(e->w) * p.n * cs;
            if (smem > smem_limit || p.in.d != 1 || p.out.d != 1 || p.in.cs != 1 || p.out.cs != 1) return;
            p.w = e->w;
            ps.smem_bytes = smem;
            // contiguous lines, columns of at most one tensor-map box: the TMA-staged variant
            ps.tma = req.use_tma && p.n <= 256 && p.in.ks * p.n == p.in.hi && p.n_outer >= 1;
        } else {
            if (rows % e->w != 0) return;
            const int64_t smem = static_cast<int64_t>(e->w) * p.pitch * cs;
            if (smem > smem_limit) return;
            // flat row index l = o * rows + k1 with pitch n
            p.n_cols = p.n_outer * p.n_cols;
            p.n_outer = 1;
            p.in.hi = 0;
            p.in.cs = p.n;
            p.in.ks = 1;
            p.ts_rows = rows;
            p.ts_line = line;
            p.w = e->w;
            ps.smem_bytes = smem;
        }
        ps.threads = threads;
        p.tpl = e->tpl;
        p.col_tiles = (p.n_cols + p.w - 1) / p.w;
        p.tiles = p.n_outer * p.col_tiles;
        ps.kc.maxt = e->maxt;
        ps.fixed_id = e->id;
        ps.fixed_feat = feat;
        use_base_table(ps);
    }

    bool fits(int64_t n, int mode) {
        SingleCfg cfg = single_cfg(n, req.dbl, req.force_maxv);
        if (!cfg.ok) return false;
        const int64_t bytes = mode == kModeK ? int64_t(kmode_pitch(static_cast<int>(n), pad_shift_for(req.dbl))) * cs
                                             : n * cs;
        return bytes <= smem_limit;
    }

    void set_fft(PassSpec&, StageSeq& seq, int* tid, int n, const SingleCfg& cfg) {
        seq = make_seq(n, cfg.radices, cfg.kc.maxv, tid);
    }

    // Choose N1 * N2 = n with both factors fitting one CTA; most balanced, N2 >= N1.
    bool split(int64_t n, int64_t& n1, int64_t& n2) {
        // a requested column length (tuning), when it divides n and both factors fit a CTA
        if (req.force_n1 > 1 && n % req.force_n1 == 0) {
            const int64_t a = req.force_n1, b = n / a;
            if (fits(a, kModeC) && fits(b, kModeK) && fits(b, kModeC)) {
                n1 = a;
                n2 = b;
                return true;
            }
        }
        int64_t best1 = 0;
        double best_score = 1e300;
        for (int64_t d = 2; d * d <= n; ++d) {
            if (n % d) continue;
            const int64_t a = d, b = n / d;
            if (!fits(a, kModeC) || !fits(b, kModeK) || !fits(b, kModeC)) continue;
            const double score = std::fabs(std::log(double(b)) - std::log(double(a)));
            if (score < best_score) { best_score = score; best1 = a; }
        }
        if (!best1) return false;
        n1 = best1;
        n2 = n / best1;
        return true;
    }

    // Chirp c_n = conj(h_n) and the convolution kernel's spectrum FFT_M(h)/M, with
    // h_n = exp(-i*sgn*pi*(n^2 mod 2L)/L) (exact reduction), h mirrored to M - n.
    void chirp_tables(int64_t L, int64_t M, int sgn, std::vector<std::complex<double>>& chirp,
                      std::vector<std::complex<double>>& kern) {
        chirp.assign(L, 0.0);
        kern.assign(M, 0.0);
        for (int64_t n = 0; n < L; ++n) {
            const uint64_t r = (static_cast<unsigned __int128>(n) * n) % static_cast<uint64_t>(2 * L);
            const std::complex<double> h = cis_neg(sgn * static_cast<int64_t>(r), 2 * L);
            kern[n] = h;
            if (n) kern[M - n] = h;
            chirp[n] = std::conj(h);
        }
        host_fft_fp64(kern, -1);
        for (auto& v : kern) v /= static_cast<double>(M);
    }

    // Stage sequence of a catalog entry (twiddles: the base table of its radices).
    StageSeq entry_seq(const BlueEntry& e) {
        StageSeq q;
        q.nstages = e.nstages;
        int ns = 1;
        for (int i = 0; i < e.nstages; ++i) {
            q.radix[i] = e.radices[i];
            q.ns[i] = ns;
            ns *= e.radices[i];
        }
        return q;
    }

    // Lines per CTA of a kModeK catalog kernel: about 256 threads, within MAXT and shared memory.
    int lines_per_cta(int tpl, int maxt, int64_t pitch, int64_t n_cols) {
        int w = std::max(1, 256 / tpl);
        w = static_cast<int>(std::min<int64_t>(w, n_cols));
        while (w > 1 && (w * tpl > maxt || static_cast<int64_t>(w) * pitch * cs > smem_limit)) --w;
        return w;
    }

    // Rader on the size-specialised Bluestein kernels (contiguous axes, prime L): with g a
    // primitive root mod L, X[g^-q] = x[0] + sum_{p<M} x[g^p] W^(g^(p-q)), M = L - 1, a cyclic
    // convolution of a[p] = x[g^p] with b[m] = W^(g^-m) (W = exp(sgn 2 pi i / L)). It runs on
    // the Bluestein kernels' Rader instantiations: the gather a[p] = x[perm_in[p]] replaces
    // the chirp pre-multiply, the scatter y[perm_out[q]] the post-multiply and truncation, and
    // bin 0 of the convolution pass gives X[0] = x[0] + sum a and adds x[0] to every output.
    // M = L - 1 instead of Bluestein's >= 2L - 2 halves the convolution; taken where the catalog
    // has a fused kernel of length M or a column x row split of it.
    bool rader_fixed(int ax, int64_t L, int64_t O, Buf& cur) {
        if (req.no_fixed || req.no_rader || L < 3 || L > (int64_t(1) << 30) || !is_prime(L)) return false;
        const int64_t M = L - 1;
        int count = 0;
        const BlueEntry* cat = blue_entries(&count);
        const int ps_shift = pad_shift_for(req.dbl);
        const BlueEntry* fused = nullptr;
        for (int i = 0; i < count && !fused; ++i) {
            const BlueEntry& e = cat[i];
            if (e.dbl == (req.dbl ? 1 : 0) && e.kind == kBlueFused && e.n == M &&
                int64_t(kmode_pitch(e.n, ps_shift)) * cs <= smem_limit)
                fused = &e;
        }
        const BlueEntry *cf = nullptr, *rc = nullptr, *ci = nullptr;
        for (int i = 0; i < count && !fused; ++i) {
            const BlueEntry& a = cat[i];
            if (a.dbl != (req.dbl ? 1 : 0) || a.kind != kBlueColsFwd || M % a.n) continue;
            if (int64_t(a.n) * a.w * cs > smem_limit) continue;
            for (int k = 0; k < count; ++k) {
                const BlueEntry& b = cat[k];
                if (b.dbl != (req.dbl ? 1 : 0) || b.kind != kBlueRowsConv || int64_t(a.n) * b.n != M) continue;
                if (int64_t(kmode_pitch(b.n, ps_shift)) * cs > smem_limit) continue;
                if (!cf || std::abs(std::log(double(b.n) / a.n)) < std::abs(std::log(double(rc->n) / cf->n))) {
                    cf = &a;
                    rc = &b;
                }
            }
        }
        if (cf)
            for (int i = 0; i < count; ++i)
                if (cat[i].dbl == cf->dbl && cat[i].kind == kBlueColsInv && cat[i].n == cf->n) ci = &cat[i];
        if (!fused && !(cf && rc && ci)) return false;

        const int sgn = req.direction;
        const int64_t E = static_cast<int64_t>(plan.elements);
        const int64_t n1 = fused ? 0 : cf->n, n2 = fused ? 0 : rc->n;
        const uint64_t g = primitive_root(static_cast<uint64_t>(L));
        const uint64_t ginv = pow_mod(g, static_cast<uint64_t>(L) - 2, static_cast<uint64_t>(L));
        std::vector<int32_t> pin(M), pout(M);
        for (uint64_t i = 0, a = 1, b = 1; i < static_cast<uint64_t>(M); ++i) {
            pin[i] = static_cast<int32_t>(a);
            pout[i] = static_cast<int32_t>(b);
            a = a * g % static_cast<uint64_t>(L);
            b = b * ginv % static_cast<uint64_t>(L);
        }
        // spectrum of b / M (the inverse FFT of the product then carries no scale); three-pass
        // plans take it permuted, K'[k1*n2 + k2] = K[k1 + n1*k2]
        auto spec = cached_table({L, M, sgn, n1, n2, -500}, [&] {
            std::vector<std::complex<double>> k(M);
            for (int64_t m = 0; m < M; ++m) k[m] = cis_neg(-int64_t(sgn) * pout[m], L);
            host_fft_fp64(k, -1);
            for (auto& v : k) v /= static_cast<double>(M);
            if (fused) return k;
            std::vector<std::complex<double>> kp(M);
            for (int64_t k1 = 0; k1 < n1; ++k1)
                for (int64_t k2 = 0; k2 < n2; ++k2) kp[k1 * n2 + k2] = k[k1 + n1 * k2];
            return kp;
        });
        const int spec_id = add_table(*spec);
        const int pin_id = add_index_table(std::move(pin));
        const int pout_id = add_index_table(std::move(pout));
        if (fused) {
            PassSpec ps;
            ps.kind = "rader_fused";
            ps.axis = ax;
            PassParams& p = ps.p;
            p.n = static_cast<int>(M);
            p.mode = kModeK;
            p.n_outer = 1;
            p.n_cols = O;
            p.in.cs = L;
            p.in.ks = 1;
            p.out = p.in;
            p.in_len = p.out_len = M;
            ps.tables.perm_in = pin_id;
            ps.tables.perm_out = pout_id;
            ps.tables.pointwise = spec_id;
            p.conj_mid = 1;
            p.conj_out = 1;
            p.fft1 = entry_seq(*fused);
            p.fft2 = p.fft1;
            use_base_table(ps);
            ps.tables.tw2 = ps.tables.tw1;
            p.pad_shift = ps_shift;
            p.pitch = kmode_pitch(p.n, ps_shift);
            p.tpl = fused->tpl;
            p.w = lines_per_cta(fused->tpl, fused->maxt, p.pitch, O);
            p.col_tiles = (p.n_cols + p.w - 1) / p.w;
            p.tiles = p.col_tiles;
            ps.threads = round_up(p.w * p.tpl, 32);
            ps.smem_bytes = static_cast<int64_t>(p.w) * p.pitch * cs;
            ps.kc.maxt = fused->maxt;
            ps.blue_id = fused->id;
            ps.blue_kind = kBlueFused;
            ps.rader = true;
            ps.src = cur;
            ps.dst = Buf::Output;
            ps.bytes_moved = 2 * E * cs;
            plan.passes.push_back(ps);
            cur = Buf::Output;
            return true;
        }
        plan.scratch_elements = std::max<uint64_t>(plan.scratch_elements, static_cast<uint64_t>(O * M));
        auto cols = [&](PassSpec& a, const BlueEntry& e) {
            PassParams& p = a.p;
            p.n = static_cast<int>(n1);
            p.mode = kModeC;
            p.g_k = n2;
            p.n_outer = O;
            p.n_cols = n2;
            p.sel_mode = kSelCol;
            p.fft1 = entry_seq(e);
            use_base_table(a);
            p.tpl = e.tpl;
            p.w = e.w;
            p.col_tiles = (p.n_cols + p.w - 1) / p.w;
            p.tiles = p.n_outer * p.col_tiles;
            a.threads = round_up(e.w * e.tpl, 32);
            a.smem_bytes = static_cast<int64_t>(e.w) * n1 * cs;
            a.kc.maxt = e.maxt;
            a.blue_id = e.id;
            a.blue_kind = e.kind;
            a.rader = true;
        };
        // pass 1: columns of the gathered line a[p] = x[g^p]; W_M^(k1*c) on the store
        PassSpec a;
        a.kind = "rader_cols_fwd";
        a.axis = ax;
        cols(a, *cf);
        a.p.in.hi = L; a.p.in.cs = 1; a.p.in.ks = n2;
        a.p.out.hi = M; a.p.out.cs = 1; a.p.out.ks = n2;
        a.p.in_len = M;
        a.p.out_len = kNoLimit;
        a.tables.perm_in = pin_id;
        add_tw4(a, M, -1);
        a.src = cur;
        a.dst = Buf::Scratch;
        a.bytes_moved = (E + O * M) * cs;
        plan.passes.push_back(a);
        // pass 2: rows: FFT, spectrum multiply (and the x[0] term, X[0] stored), inverse FFT,
        // inverse twiddle, in place
        PassSpec b;
        b.kind = "rader_rows_conv";
        b.axis = ax;
        {
            PassParams& p = b.p;
            p.n = static_cast<int>(n2);
            p.mode = kModeK;
            p.n_outer = 1;
            p.n_cols = O * n1;
            p.in.cs = n2;
            p.in.ks = 1;
            p.out = p.in;
            p.sel_mode = kSelColMod;
            p.sel_d = n1;
            p.in_len = p.out_len = kNoLimit;
            b.tables.pointwise = spec_id;
            p.pw_stride = n2;
            p.conj_mid = 1;
            p.conj_out = 1;
            p.fft1 = entry_seq(*rc);
            p.fft2 = p.fft1;
            use_base_table(b);
            b.tables.tw2 = b.tables.tw1;
            add_tw4(b, M, +1);
            p.pad_shift = ps_shift;
            p.pitch = kmode_pitch(p.n, ps_shift);
            p.tpl = rc->tpl;
            p.w = lines_per_cta(rc->tpl, rc->maxt, p.pitch, p.n_cols);
            p.col_tiles = (p.n_cols + p.w - 1) / p.w;
            p.tiles = p.col_tiles;
            b.threads = round_up(p.w * p.tpl, 32);
            b.smem_bytes = static_cast<int64_t>(p.w) * p.pitch * cs;
            b.kc.maxt = rc->maxt;
            b.blue_id = rc->id;
            b.blue_kind = kBlueRowsConv;
            b.rader = true;
            b.rader_dc = true;
            b.rader_src = cur;
            b.src = Buf::Scratch;
            b.dst = Buf::Scratch;
            b.bytes_moved = 2 * O * M * cs;
        }
        plan.passes.push_back(b);
        // pass 3: columns: inverse FFT, scatter y[g^-q] (positions 1 .. L-1)
        PassSpec c;
        c.kind = "rader_cols_inv";
        c.axis = ax;
        cols(c, *ci);
        c.p.in.hi = M; c.p.in.cs = 1; c.p.in.ks = n2;
        c.p.out.hi = L; c.p.out.cs = 1; c.p.out.ks = n2;
        c.p.in_len = kNoLimit;
        c.p.out_len = M;
        c.p.conj_in = 1;
        c.p.conj_out = 1;
        c.tables.perm_out = pout_id;
        c.smem_bytes += static_cast<int64_t>(ci->w) * n1 * static_cast<int64_t>(sizeof(int32_t));  // scatter indices
        c.src = Buf::Scratch;
        c.dst = Buf::Output;
        c.bytes_moved = (O * M + E) * cs;
        plan.passes.push_back(c);
        cur = Buf::Output;
        return true;
    }

    // Bluestein on the size-specialised kernels (contiguous axes): the smallest catalog
    // convolution length M >= 2L - 2 (bluestein_length), as one fused pass where a fused
    // kernel of length M fits a CTA, else as M = n1 * n2 over a column kernel (n1) and a row
    // kernel (n2) in three passes. Returns false (generic kernels) when the catalog has no such length.
    bool bluestein_fixed(int ax, int64_t L, int64_t O, Buf& cur) {
        if (req.no_fixed) return false;
        int count = 0;
        const BlueEntry* cat = blue_entries(&count);
        const int64_t need = 2 * L - 2;
        const int ps_shift = pad_shift_for(req.dbl);
        const BlueEntry* fused = nullptr;
        for (int i = 0; i < count; ++i) {
            const BlueEntry& e = cat[i];
            if (e.dbl != (req.dbl ? 1 : 0) || e.kind != kBlueFused || e.n < need) continue;
            if (int64_t(kmode_pitch(e.n, ps_shift)) * cs > smem_limit) continue;
            if (!fused || e.n < fused->n) fused = &e;
        }
        const BlueEntry *cf = nullptr, *rc = nullptr;
        int64_t best = 0;
        for (int i = 0; i < count && !fused; ++i) {
            const BlueEntry& a = cat[i];
            if (a.dbl != (req.dbl ? 1 : 0) || a.kind != kBlueColsFwd) continue;
            if (int64_t(a.n) * a.w * cs > smem_limit) continue;
            for (int k = 0; k < count; ++k) {
                const BlueEntry& b = cat[k];
                if (b.dbl != (req.dbl ? 1 : 0) || b.kind != kBlueRowsConv) continue;
                const int64_t M = int64_t(a.n) * b.n;
                if (M < need || int64_t(kmode_pitch(b.n, ps_shift)) * cs > smem_limit) continue;
                const bool better = !cf || M < best ||
                                    (M == best && std::abs(std::log(double(b.n) / a.n)) <
                                                      std::abs(std::log(double(rc->n) / cf->n)));
                if (better) {
                    best = M;
                    cf = &a;
                    rc = &b;
                }
            }
        }
        const BlueEntry* ci = nullptr;
        if (cf)
            for (int i = 0; i < count; ++i)
                if (cat[i].dbl == cf->dbl && cat[i].kind == kBlueColsInv && cat[i].n == cf->n) ci = &cat[i];
        if (!fused && !(cf && rc && ci)) return false;

        const bool bwd = req.direction == 1;
        (void)bwd;
        const int sgn = req.direction;
        const int64_t E = static_cast<int64_t>(plan.elements);
        const int64_t M = fused ? fused->n : best;
        std::vector<std::complex<double>> chirp, kern;
        if (!req.device_spectrum) chirp_tables(L, M, sgn, chirp, kern);
        const int chirp_id = req.device_spectrum ? add_device_table(L) : add_table(std::move(chirp));
        BluesteinJob job;
        job.L = L;
        job.M = M;
        job.sgn = sgn;
        job.chirp_table = chirp_id;
        if (fused) {
            PassSpec ps;
            ps.kind = "bluestein_fused";
            ps.axis = ax;
            PassParams& p = ps.p;
            p.n = static_cast<int>(M);
            p.mode = kModeK;
            p.n_outer = 1;
            p.n_cols = O;
            p.in.cs = L;
            p.in.ks = 1;
            p.out = p.in;
            p.in_len = p.out_len = L;
            ps.tables.premul = chirp_id;
            ps.tables.postmul = chirp_id;
            ps.tables.pointwise = req.device_spectrum ? add_device_table(M) : add_table(std::move(kern));
            job.spectrum_table = ps.tables.pointwise;
            p.conj_mid = 1;
            p.conj_out = 1;
            p.fft1 = entry_seq(*fused);
            p.fft2 = p.fft1;
            use_base_table(ps);
            ps.tables.tw2 = ps.tables.tw1;
            p.pad_shift = ps_shift;
            p.pitch = kmode_pitch(p.n, ps_shift);
            p.tpl = fused->tpl;
            p.w = lines_per_cta(fused->tpl, fused->maxt, p.pitch, O);
            p.col_tiles = (p.n_cols + p.w - 1) / p.w;
            p.tiles = p.col_tiles;
            ps.threads = round_up(p.w * p.tpl, 32);
            ps.smem_bytes = static_cast<int64_t>(p.w) * p.pitch * cs;
            ps.kc.maxt = fused->maxt;
            ps.blue_id = fused->id;
            ps.blue_kind = kBlueFused;
            ps.src = cur;
            ps.dst = Buf::Output;
            ps.bytes_moved = 2 * E * cs;
            plan.passes.push_back(ps);
            if (req.device_spectrum) plan.bluestein_jobs.push_back(job);
            cur = Buf::Output;
            return true;
        }
        const int64_t n1 = cf->n, n2 = rc->n;
        int kp_id;
        if (!req.device_spectrum) {
            std::vector<std::complex<double>> kp(M);  // K'[k1*n2 + k2] = K[k1 + n1*k2]
            for (int64_t k1 = 0; k1 < n1; ++k1)
                for (int64_t k2 = 0; k2 < n2; ++k2) kp[k1 * n2 + k2] = kern[k1 + n1 * k2];
            kp_id = add_table(std::move(kp));
        } else {
            kp_id = add_device_table(M);
            job.n1 = n1;
            job.n2 = n2;
            job.large = true;
            job.spectrum_table = kp_id;
            plan.bluestein_jobs.push_back(job);
        }
        plan.scratch_elements = std::max<uint64_t>(plan.scratch_elements, static_cast<uint64_t>(O * M));
        auto cols = [&](PassSpec& a, const BlueEntry& e) {
            PassParams& p = a.p;
            p.n = static_cast<int>(n1);
            p.mode = kModeC;
            p.g_k = n2;
            p.n_outer = O;
            p.n_cols = n2;
            p.sel_mode = kSelCol;
            p.fft1 = entry_seq(e);
            use_base_table(a);
            p.tpl = e.tpl;
            p.w = e.w;
            p.col_tiles = (p.n_cols + p.w - 1) / p.w;
            p.tiles = p.n_outer * p.col_tiles;
            a.threads = round_up(e.w * e.tpl, 32);
            a.smem_bytes = static_cast<int64_t>(e.w) * n1 * cs;
            a.kc.maxt = e.maxt;
            a.blue_id = e.id;
            a.blue_kind = e.kind;
        };
        // pass 1: columns of the zero-padded, chirp-multiplied line; W_M^(k1*c) on the store
        PassSpec a;
        a.kind = "bluestein_cols_fwd";
        a.axis = ax;
        cols(a, *cf);
        a.p.in.hi = L; a.p.in.cs = 1; a.p.in.ks = n2;
        a.p.out.hi = M; a.p.out.cs = 1; a.p.out.ks = n2;
        a.p.in_len = L;
        a.p.out_len = kNoLimit;
        a.tables.premul = chirp_id;
        add_tw4(a, M, -1);
        a.src = cur;
        a.dst = Buf::Scratch;
        a.bytes_moved = (E + O * M) * cs;
        plan.passes.push_back(a);
        // pass 2: rows (all lines' rows in one flat range): FFT, spectrum multiply, inverse
        // FFT, inverse twiddle, in place
        PassSpec b;
        b.kind = "bluestein_rows_conv";
        b.axis = ax;
        {
            PassParams& p = b.p;
            p.n = static_cast<int>(n2);
            p.mode = kModeK;
            p.n_outer = 1;
            p.n_cols = O * n1;
            p.in.cs = n2;
            p.in.ks = 1;
            p.out = p.in;
            p.sel_mode = kSelColMod;
            p.sel_d = n1;
            p.in_len = p.out_len = kNoLimit;
            b.tables.pointwise = kp_id;
            p.pw_stride = n2;
            p.conj_mid = 1;
            p.conj_out = 1;
            p.fft1 = entry_seq(*rc);
            p.fft2 = p.fft1;
            use_base_table(b);
            b.tables.tw2 = b.tables.tw1;
            add_tw4(b, M, +1);
            p.pad_shift = ps_shift;
            p.pitch = kmode_pitch(p.n, ps_shift);
            p.tpl = rc->tpl;
            p.w = lines_per_cta(rc->tpl, rc->maxt, p.pitch, p.n_cols);
            p.col_tiles = (p.n_cols + p.w - 1) / p.w;
            p.tiles = p.col_tiles;
            b.threads = round_up(p.w * p.tpl, 32);
            b.smem_bytes = static_cast<int64_t>(p.w) * p.pitch * cs;
            b.kc.maxt = rc->maxt;
            b.blue_id = rc->id;
            b.blue_kind = kBlueRowsConv;
            b.src = Buf::Scratch;
            b.dst = Buf::Scratch;
            b.bytes_moved = 2 * O * M * cs;
        }
        plan.passes.push_back(b);
        // pass 3: columns: inverse FFT, chirp post-multiply, truncation to L
        PassSpec c;
        c.kind = "bluestein_cols_inv";
        c.axis = ax;
        cols(c, *ci);
        c.p.in.hi = M; c.p.in.cs = 1; c.p.in.ks = n2;
        c.p.out.hi = L; c.p.out.cs = 1; c.p.out.ks = n2;
        c.p.in_len = kNoLimit;
        c.p.out_len = L;
        c.p.conj_in = 1;
        c.p.conj_out = 1;
        c.tables.postmul = chirp_id;
        c.src = Buf::Scratch;
        c.dst = Buf::Output;
        c.bytes_moved = (O * M + E) * cs;
        plan.passes.push_back(c);
        cur = Buf::Output;
        return true;
    }

    // A four-step split of L whose column and row passes have size-specialised kernels that a
    // fused four-step kernel (fused4_catalog.h) runs together.
    bool fused_split(int64_t L, int64_t& n1, int64_t& n2) {
        for (int64_t a = 2; a * 2 <= L; ++a) {
            if (L % a) continue;
            const int64_t b = L / a;
            const FixedEntry* c = find_fixed(req.dbl, kModeC, static_cast<int>(a), kFixedTw4);
            const FixedEntry* r = find_fixed(req.dbl, kModeK, static_cast<int>(b), kFixedTStore);
            if (c && r && has_fused4(req.dbl, c->id, r->id)) {
                n1 = a;
                n2 = b;
                return true;
            }
        }
        return false;
    }

    void axis(int ax, int64_t L, int64_t s, int64_t O, Buf& cur) {
        const bool bwd = req.direction == 1;
        const int64_t E = static_cast<int64_t>(plan.elements);
        int64_t f1 = 0, f2 = 0;
        const bool fused_instead = s == 1 && req.fused_single && !req.no_fixed && O >= 3 && fused_split(L, f1, f2);
        if (smooth7(static_cast<uint64_t>(L))) {
            const int mode = s == 1 ? kModeK : kModeC;
            if (fits(L, mode) && !fused_instead) {
                PassSpec ps;
                ps.kind = "single";
                ps.axis = ax;
                PassParams& p = ps.p;
                p.n = static_cast<int>(L);
                p.mode = mode;
                if (s == 1) {
                    p.n_outer = 1; p.n_cols = O;
                    p.in.cs = L; p.in.ks = 1;
                } else {
                    p.n_outer = O; p.n_cols = s;
                    p.in.hi = L * s; p.in.cs = 1; p.in.ks = s;
                }
                p.out = p.in;
                p.in_len = p.out_len = L;
                p.conj_in = p.conj_out = bwd;
                SingleCfg cfg = single_cfg(L, req.dbl, req.force_maxv);
                set_fft(ps, p.fft1, &ps.tables.tw1, p.n, cfg);
                geometry(ps, cfg, req.force_w);
                try_fixed(ps, cfg);
                if (req.split_bf16) try_tc(ps);
                ps.src = cur;
                ps.dst = Buf::Output;
                ps.bytes_moved = 2 * E * cs;
                plan.passes.push_back(ps);
                cur = Buf::Output;
                return;
            }
            // The cluster kernel is opt-in (cluster_p > 0, chosen by the autotuner or the caller):
            // measured slower than the size-specialised two-pass four-step on B200.
            if (s == 1 && !req.no_cluster && req.cluster_p > 0) {
                if (const ClusterEntry* ce = find_cluster(req.dbl, L, req.cluster_p)) {
                    cluster_pass(ax, L, O, *ce, cur);
                    return;
                }
            }
            int64_t n1, n2;
            if (fused_instead) {
                n1 = f1;
                n2 = f2;
            } else if (!split(L, n1, n2)) {
                throw std::runtime_error("FFT length too large for this provider");
            }
            plan.scratch_elements = std::max<uint64_t>(plan.scratch_elements, static_cast<uint64_t>(E));
            // column pass
            PassSpec a;
            a.kind = "fourstep_cols";
            a.axis = ax;
            {
                PassParams& p = a.p;
                p.n = static_cast<int>(n1);
                p.mode = kModeC;
                p.g_k = n2;
                if (s == 1) {
                    p.n_outer = O; p.n_cols = n2;
                    p.in.hi = L; p.in.cs = 1; p.in.ks = n2;
                    p.sel_mode = kSelCol;
                } else {
                    p.n_outer = O * n2; p.n_cols = s;
                    p.in.hi = L * s; p.in.d = n2; p.in.lo = s; p.in.cs = 1; p.in.ks = n2 * s;
                    p.sel_mode = kSelOuterLo; p.sel_d = n2;
                }
                p.out = p.in;
                p.in_len = p.out_len = L;
                p.conj_in = bwd;
                SingleCfg cfg = single_cfg(n1, req.dbl, req.force_maxv);
                set_fft(a, p.fft1, &a.tables.tw1, p.n, cfg);
                add_tw4(a, L, -1);
                geometry(a, cfg, s == 1 ? fourstep_w(cfg.tpl, req.dbl ? 8 : 16) : 0);
                if (s == 1) try_fixed_fourstep(a, kFixedTw4);
                a.src = cur;
                a.dst = Buf::Scratch;
                a.bytes_moved = 2 * E * cs;
            }
            plan.passes.push_back(a);
            PassSpec b;
            b.kind = "fourstep_rows";
            b.axis = ax;
            {
                PassParams& p = b.p;
                p.n = static_cast<int>(n2);
                if (s == 1) {
                    p.mode = kModeK;
                    p.n_outer = O; p.n_cols = n1;
                    p.in.hi = L; p.in.cs = n2; p.in.ks = 1;
                    p.out.hi = L; p.out.cs = 1; p.out.ks = n1;
                    p.store_via_smem = 1;
                } else {
                    p.mode = kModeC;
                    p.n_outer = O * n1; p.n_cols = s;
                    p.in.hi = L * s; p.in.d = n1; p.in.lo = n2 * s; p.in.cs = 1; p.in.ks = s;
                    p.out.hi = L * s; p.out.d = n1; p.out.lo = s; p.out.cs = 1; p.out.ks = n1 * s;
                }
                p.in_len = p.out_len = kNoLimit;
                p.conj_out = bwd;
                SingleCfg cfg = single_cfg(n2, req.dbl, req.force_maxv);
                set_fft(b, p.fft1, &b.tables.tw1, p.n, cfg);
                // rows per CTA: enough for 128-byte segments of the transposed store
                geometry(b, cfg, s == 1 ? fourstep_w(cfg.tpl, std::max(1, 128 / cs)) : 0);
                if (s == 1) try_fixed_fourstep(b, kFixedTStore, n1, L);
                b.src = Buf::Scratch;
                b.dst = Buf::Output;
                b.bytes_moved = 2 * E * cs;
            }
            plan.passes.push_back(b);
            cur = Buf::Output;
            return;
        }

        if (s == 1 && rader_fixed(ax, L, O, cur)) return;
        if (s == 1 && bluestein_fixed(ax, L, O, cur)) return;
        // Bluestein: y_k = c_k * sum_n (x_n c_n) h_{k-n}, c_n = exp(-i*sgn*pi*n^2/L) conj-chirp,
        // h_n = conj(c_n) (exact n^2 mod 2L reduction), convolution of length M via FFT.
        const int64_t M = static_cast<int64_t>(bluestein_length(static_cast<uint64_t>(L)));
        const int sgn = req.direction;  // -1 forward, +1 backward
        std::vector<std::complex<double>> chirp, kern;
        if (!req.device_spectrum) {
            chirp.assign(L, 0.0);
            kern.assign(M, 0.0);
            for (int64_t n = 0; n < L; ++n) {
                const uint64_t r = (static_cast<unsigned __int128>(n) * n) % static_cast<uint64_t>(2 * L);
                // h_n = exp(-i*sgn*pi*r/L) = exp(-2 pi i * (sgn*r) / (2L))
                const std::complex<double> h = cis_neg(sgn * static_cast<int64_t>(r), 2 * L);
                kern[n] = h;
                if (n) kern[M - n] = h;
                chirp[n] = std::conj(h);
            }
            host_fft_fp64(kern, -1);
            for (auto& v : kern) v /= static_cast<double>(M);
        }
        const int chirp_id = req.device_spectrum ? add_device_table(L) : add_table(std::move(chirp));
        const int mode = s == 1 ? kModeK : kModeC;
        if (fits(M, mode)) {
            PassSpec ps;
            ps.kind = "bluestein_fused";
            ps.axis = ax;
            PassParams& p = ps.p;
            p.n = static_cast<int>(M);
            p.mode = mode;
            if (s == 1) {
                p.n_outer = 1; p.n_cols = O;
                p.in.cs = L; p.in.ks = 1;
            } else {
                p.n_outer = O; p.n_cols = s;
                p.in.hi = L * s; p.in.cs = 1; p.in.ks = s;
            }
            p.out = p.in;
            p.in_len = p.out_len = L;
            ps.tables.premul = chirp_id;
            ps.tables.postmul = chirp_id;
            ps.tables.pointwise = req.device_spectrum ? add_device_table(M) : add_table(std::move(kern));
            if (req.device_spectrum) {
                BluesteinJob job;
                job.L = L;
                job.M = M;
                job.sgn = sgn;
                job.chirp_table = chirp_id;
                job.spectrum_table = ps.tables.pointwise;
                plan.bluestein_jobs.push_back(job);
            }
            p.conj_mid = 1;
            p.conj_out = 1;
            SingleCfg cfg = single_cfg(M, req.dbl, req.force_maxv);
            set_fft(ps, p.fft1, &ps.tables.tw1, p.n, cfg);
            set_fft(ps, p.fft2, &ps.tables.tw2, p.n, cfg);
            geometry(ps, cfg, req.force_w);
            ps.src = cur;
            ps.dst = Buf::Output;
            ps.bytes_moved = 2 * E * cs;
            plan.passes.push_back(ps);
            cur = Buf::Output;
            return;
        }
        int64_t n1, n2;
        if (!split(M, n1, n2)) throw std::runtime_error("Bluestein length too large for this provider");
        // K'[k1*N2 + k2] = K[k1 + N1*k2]
        int kp_id;
        if (!req.device_spectrum) {
            std::vector<std::complex<double>> kp(M);
            for (int64_t k1 = 0; k1 < n1; ++k1)
                for (int64_t k2 = 0; k2 < n2; ++k2) kp[k1 * n2 + k2] = kern[k1 + n1 * k2];
            kp_id = add_table(std::move(kp));
        } else {
            kp_id = add_device_table(M);
        }
        if (req.device_spectrum) {
            BluesteinJob job;
            job.L = L;
            job.M = M;
            job.n1 = n1;
            job.n2 = n2;
            job.sgn = sgn;
            job.large = true;
            job.chirp_table = chirp_id;
            job.spectrum_table = kp_id;
            plan.bluestein_jobs.push_back(job);
        }
        const int64_t lines = E / L;
        plan.scratch_elements = std::max<uint64_t>(plan.scratch_elements, static_cast<uint64_t>(lines * M));
        // pass 1: columns of the zero-padded, chirp-multiplied line
        PassSpec a;
        a.kind = "bluestein_cols_fwd";
        a.axis = ax;
        {
            PassParams& p = a.p;
            p.n = static_cast<int>(n1);
            p.mode = kModeC;
            p.g_k = n2;
            if (s == 1) {
                p.n_outer = O; p.n_cols = n2;
                p.in.hi = L; p.in.cs = 1; p.in.ks = n2;
                p.out.hi = M; p.out.cs = 1; p.out.ks = n2;
                p.sel_mode = kSelCol;
            } else {
                p.n_outer = O * n2; p.n_cols = s;
                p.in.hi = L * s; p.in.d = n2; p.in.lo = s; p.in.cs = 1; p.in.ks = n2 * s;
                p.out.hi = M * s; p.out.d = n2; p.out.lo = s; p.out.cs = 1; p.out.ks = n2 * s;
                p.sel_mode = kSelOuterLo; p.sel_d = n2;
            }
            p.in_len = L;
            p.out_len = kNoLimit;
            a.tables.premul = chirp_id;
            SingleCfg cfg = single_cfg(n1, req.dbl, req.force_maxv);
            set_fft(a, p.fft1, &a.tables.tw1, p.n, cfg);
            add_tw4(a, M, -1);
            geometry(a, cfg, 0);
            a.src = cur;
            a.dst = Buf::Scratch;
            a.bytes_moved = (E + lines * M) * cs;
        }
        plan.passes.push_back(a);
        // pass 2: rows: FFT, spectrum multiply, inverse FFT, inverse twiddle
        PassSpec b;
        b.kind = "bluestein_rows_conv";
        b.axis = ax;
        {
            PassParams& p = b.p;
            p.n = static_cast<int>(n2);
            if (s == 1) {
                p.mode = kModeK;
                p.n_outer = O; p.n_cols = n1;
                p.in.hi = M; p.in.cs = n2; p.in.ks = 1;
                p.sel_mode = kSelCol;
            } else {
                p.mode = kModeC;
                p.n_outer = O * n1; p.n_cols = s;
                p.in.hi = M * s; p.in.d = n1; p.in.lo = n2 * s; p.in.cs = 1; p.in.ks = s;
                p.sel_mode = kSelOuterLo; p.sel_d = n1;
            }
            p.out = p.in;
            p.in_len = p.out_len = kNoLimit;
            b.tables.pointwise = kp_id;
            p.pw_stride = n2;
            p.conj_mid = 1;
            p.conj_out = 1;
            SingleCfg cfg = single_cfg(n2, req.dbl, req.force_maxv);
            set_fft(b, p.fft1, &b.tables.tw1, p.n, cfg);
            set_fft(b, p.fft2, &b.tables.tw2, p.n, cfg);
            add_tw4(b, M, +1);
            geometry(b, cfg, 0);
            b.src = Buf::Scratch;
            b.dst = Buf::Scratch;
            b.bytes_moved = 2 * lines * M * cs;
        }
        plan.passes.push_back(b);
        // pass 3: columns: inverse FFT, chirp post-multiply, truncation to L
        PassSpec c;
        c.kind = "bluestein_cols_inv";
        c.axis = ax;
        {
            PassParams& p = c.p;
            p.n = static_cast<int>(n1);
            p.mode = kModeC;
            p.g_k = n2;
            if (s == 1) {
                p.n_outer = O; p.n_cols = n2;
                p.in.hi = M; p.in.cs = 1; p.in.ks = n2;
                p.out.hi = L; p.out.cs = 1; p.out.ks = n2;
                p.sel_mode = kSelCol;
            } else {
                p.n_outer = O * n2; p.n_cols = s;
                p.in.hi = M * s; p.in.d = n2; p.in.lo = s; p.in.cs = 1; p.in.ks = n2 * s;
                p.out.hi = L * s; p.out.d = n2; p.out.lo = s; p.out.cs = 1; p.out.ks = n2 * s;
                p.sel_mode = kSelOuterLo; p.sel_d = n2;
            }
            p.in_len = kNoLimit;
            p.out_len = L;
            p.conj_in = 1;
            p.conj_out = 1;
            c.tables.postmul = chirp_id;
            SingleCfg cfg = single_cfg(n1, req.dbl, req.force_maxv);
            set_fft(c, p.fft1, &c.tables.tw1, p.n, cfg);
            geometry(c, cfg, 0);
            c.src = Buf::Scratch;
            c.dst = Buf::Output;
            c.bytes_moved = (lines * M + E) * cs;
        }
        plan.passes.push_back(c);
        cur = Buf::Output;
    }

    // Whole line of length L = n1*n2 on one thread-block cluster (single HBM round trip).
    void cluster_pass(int ax, int64_t L, int64_t O, const ClusterEntry& ce, Buf& cur) {
        PassSpec ps;
        ps.kind = "cluster";
        ps.axis = ax;
        PassParams& p = ps.p;
        p.n = static_cast<int>(L);
        p.mode = kModeK;
        p.n_outer = 1;
        p.n_cols = O;
        p.in.cs = L; p.in.ks = 1;
        p.out = p.in;
        p.in_len = p.out_len = L;
        p.conj_in = p.conj_out = req.direction == 1;
        std::vector<int> r1(ce.r1, ce.r1 + ce.ns1), r2(ce.r2, ce.r2 + ce.ns2);
        p.fft1 = make_seq(ce.n1, r1, 0, &ps.tables.tw1);
        p.fft2 = make_seq(ce.n2, r2, 0, &ps.tables.tw2);
        add_tw4(ps, L, -1);
        ps.cluster_id = ce.id;
        ps.cl_n1 = ce.n1;
        ps.cl_n2 = ce.n2;
        ps.cl_p = ce.p;
        if (req.cluster_pipe && req.dbl && L == 65536 && ce.n1 == 256 && ce.n2 == 256 && ce.p == 16 &&
            r1 == std::vector<int>{8, 8, 4} && r2 == r1) {
            ps.cluster_pipe = true;
            ps.tables.cl_base = base_table(r1);
        }
        const int cw = ce.n2 / ce.p, rw = ce.n1 / ce.p;
        ps.threads = std::max(cw * ce.tpl1, rw * ce.tpl2);
        ps.smem_bytes = L / ce.p * cs;
        if (ps.smem_bytes > smem_limit) throw std::runtime_error("cluster pass exceeds shared memory");
        ps.kc.maxt = ce.maxt;
        p.w = 1;
        p.col_tiles = O;
        p.tiles = O * ce.p;
        ps.src = cur;
        ps.dst = Buf::Output;
        ps.bytes_moved = 2 * static_cast<int64_t>(plan.elements) * cs;
        plan.passes.push_back(ps);
        cur = Buf::Output;
    }

    void copy_pass(Buf& cur) {
        PassSpec ps;
        ps.kind = "copy";
        PassParams& p = ps.p;
        p.n = 1;
        p.mode = kModeK;
        p.n_outer = 1;
        p.n_cols = static_cast<int64_t>(plan.elements);
        p.in.cs = 1; p.in.ks = 1;
        p.out = p.in;
        p.in_len = p.out_len = 1;
        SingleCfg cfg;
        cfg.ok = true;
        cfg.kc.maxv = req.dbl ? 8 : 16;
        cfg.radices = {1};
        cfg.tpl = 1;
        set_fft(ps, p.fft1, &ps.tables.tw1, 1, cfg);
        geometry(ps, cfg, 256);
        ps.src = cur;
        ps.dst = Buf::Output;
        ps.bytes_moved = 2 * static_cast<int64_t>(plan.elements) * cs;
        plan.passes.push_back(ps);
        cur = Buf::Output;
    }
};

template <class... A>
constexpr int count_args(A...) {
    return static_cast<int>(sizeof...(A));
}
#define SFB_ENTRY(ID, DBL, MODEC, FEAT, N, TPL, W, MAXT, ...) \
    FixedEntry{ID, DBL, MODEC, FEAT, N, TPL, W, MAXT, {__VA_ARGS__}, count_args(__VA_ARGS__)},
const FixedEntry kFixed[] = {SFB_FIXED_CATALOG(SFB_ENTRY)};
#undef SFB_ENTRY

long double two_pi_l() { return 6.283185307179586476925286766559005768L; }

}  // namespace

uint64_t checked_element_count(const std::vector<uint64_t>& shape, uint64_t batch) {
    if (shape.empty() || shape.size() > 3) throw std::invalid_argument("FFT rank must be between 1 and 3");
    if (batch == 0) throw std::invalid_argument("FFT batch count must be non-zero");
    uint64_t count = batch;
    for (uint64_t len : shape) {
        if (len == 0) throw std::invalid_argument("FFT dimensions must be non-zero");
        if (count > std::numeric_limits<uint64_t>::max() / len)
            throw std::invalid_argument("FFT element count overflows size_t");
        count *= len;
    }
    return count;
}

double normalization_scale(int mode, int direction, uint64_t n) {
    switch (mode) {
        case 0: return 1.0;
        case 1: return direction == -1 ? 1.0 / static_cast<double>(n) : 1.0;
        case 2: return direction == 1 ? 1.0 / static_cast<double>(n) : 1.0;
        case 3: return 1.0 / std::sqrt(static_cast<double>(n));
        default: return 1.0;
    }
}

uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t m) {
    unsigned __int128 r = 1, x = b % m;
    for (; e; e >>= 1) {
        if (e & 1) r = r * x % m;
        x = x * x % m;
    }
    return static_cast<uint64_t>(r);
}

bool is_prime(uint64_t n) {
    if (n < 2) return false;
    for (uint64_t d = 2; d * d <= n; ++d)
        if (n % d == 0) return false;
    return true;
}

// Smallest generator of the multiplicative group mod a prime p: g^((p-1)/q) != 1 for every
// prime factor q of p - 1.
uint64_t primitive_root(uint64_t p) {
    if (p == 2) return 1;
    std::vector<uint64_t> qs;
    uint64_t m = p - 1;
    for (uint64_t d = 2; d * d <= m; ++d) {
        if (m % d) continue;
        qs.push_back(d);
        while (m % d == 0) m /= d;
    }
    if (m > 1) qs.push_back(m);
    for (uint64_t g = 2; g < p; ++g) {
        bool ok = true;
        for (uint64_t q : qs) ok = ok && pow_mod(g, (p - 1) / q, p) != 1;
        if (ok) return g;
    }
    throw std::invalid_argument("no primitive root");
}

bool smooth7(uint64_t n) {
    Factors f;
    return factor7(n, f);
}

// The cyclic convolution y[k] = sum_n a[n] b[k - n], k, n in [0, L), reads the chirp b at
// d = k - n in [-(L-1), L-1]. A cyclic length M keeps those reads apart except where two of
// them differ by M; for M = 2L - 2 the only such pair is d = L-1 and d = -(L-1), and the chirp
// b[d] = exp(i pi d^2 / L) is even, so both read the same value: M >= 2L - 2 is exact (one less
// than the usual 2L - 1, which makes M = 2^17 for L = 65537 instead of 163840).
uint64_t bluestein_length(uint64_t len) {
    if (len > (uint64_t(1) << 40)) throw std::invalid_argument("Bluestein convolution size overflows");
    uint64_t m = 2 * len - 2;
    while (!smooth7(m)) ++m;
    return m;
}

std::vector<int> choose_radices(int n, int maxv) {
    Factors f;
    if (!factor7(static_cast<uint64_t>(n), f)) throw std::invalid_argument("length is not 7-smooth");
    std::vector<int> r;
    if (maxv >= 16)
        while (f.e2 >= 4) { r.push_back(16); f.e2 -= 4; }
    while (f.e2 >= 3) { r.push_back(8); f.e2 -= 3; }
    if (f.e2 == 2) r.push_back(4);
    if (f.e2 == 1) r.push_back(2);
    for (int i = 0; i < f.e3; ++i) r.push_back(3);
    for (int i = 0; i < f.e5; ++i) r.push_back(5);
    for (int i = 0; i < f.e7; ++i) r.push_back(7);
    if (r.empty()) r.push_back(1);
    return r;
}

int threads_per_line(int n, const std::vector<int>& radices, int maxv) {
    int tpl = 1;
    for (int R : radices) {
        const int per = std::max(1, maxv / R);
        const int nr = n / R;
        tpl = std::max(tpl, (nr + per - 1) / per);
    }
    return tpl;
}

std::complex<double> cis_neg(int64_t num, int64_t den) {
    // exp(-2 pi i m / den) with the argument reduced to |x| <= 1/4 turn-halves by symmetry:
    // x = 2m/den in [0, 2) -> [-1, 1) -> quadrant folding, so cos/sin see |angle| <= pi/4.
    int64_t m = num % den;
    if (m < 0) m += den;
    // work in units of 1/(4 den) of a half-turn: t = 8m / den eighths
    const int64_t m8 = 8 * m;
    const int64_t oct = m8 / den;                      // 0..7 octant of the full turn
    const int64_t rem = m8 - oct * den;                // remainder in [0, den)
    const double f = static_cast<double>(rem) / static_cast<double>(den);  // [0,1) of an octant
    const double pi4 = 0.78539816339744830961566084581987572;
    double c, sn;
    // angle within the octant pair: theta = (oct + f) * pi/4
    switch (oct) {
        case 0: c = std::cos(f * pi4); sn = std::sin(f * pi4); break;
        case 1: c = std::sin((1 - f) * pi4); sn = std::cos((1 - f) * pi4); break;
        case 2: c = -std::sin(f * pi4); sn = std::cos(f * pi4); break;
        case 3: c = -std::cos((1 - f) * pi4); sn = std::sin((1 - f) * pi4); break;
        case 4: c = -std::cos(f * pi4); sn = -std::sin(f * pi4); break;
        case 5: c = -std::sin((1 - f) * pi4); sn = -std::cos((1 - f) * pi4); break;
        case 6: c = std::sin(f * pi4); sn = -std::cos(f * pi4); break;
        default: c = std::cos((1 - f) * pi4); sn = -std::sin((1 - f) * pi4); break;
    }
    (void)two_pi_l;
    return {c, -sn};
}

void host_fft_fp64(std::vector<std::complex<double>>& a, int sign) {
    const int64_t n = static_cast<int64_t>(a.size());
    if (n <= 1) return;
    Factors f;
    if (!factor7(static_cast<uint64_t>(n), f)) throw std::invalid_argument("host FFT length is not 7-smooth");
    std::vector<int> radices;
    for (int i = 0; i < f.e2; ++i) radices.push_back(2);
    for (int i = 0; i < f.e3; ++i) radices.push_back(3);
    for (int i = 0; i < f.e5; ++i) radices.push_back(5);
    for (int i = 0; i < f.e7; ++i) radices.push_back(7);
    std::vector<std::complex<double>> y(n);
    int64_t ns = 1;
    for (int R : radices) {
        const int64_t nr = n / R;
        std::vector<std::complex<double>> dft(R * R);
        for (int p = 0; p < R; ++p)
            for (int q = 0; q < R; ++q) {
                auto w = cis_neg(int64_t(p) * q, R);
                dft[p * R + q] = sign < 0 ? w : std::conj(w);
            }
        std::vector<std::complex<double>> tw(ns * R);
        for (int64_t jm = 0; jm < ns; ++jm)
            for (int r = 0; r < R; ++r) {
                auto w = cis_neg(int64_t(r) * jm, ns * R);
                tw[jm * R + r] = sign < 0 ? w : std::conj(w);
            }
        std::complex<double> v[7], u[7];
        for (int64_t j = 0; j < nr; ++j) {
            const int64_t jm = j % ns;
            for (int r = 0; r < R; ++r) v[r] = a[j + r * nr] * tw[jm * R + r];
            for (int p = 0; p < R; ++p) {
                std::complex<double> acc = 0.0;
                for (int q = 0; q < R; ++q) acc += dft[p * R + q] * v[q];
                u[p] = acc;
            }
            const int64_t base = (j - jm) * R + jm;
            for (int r = 0; r < R; ++r) y[base + r * ns] = u[r];
        }
        a.swap(y);
        ns *= R;
    }
}

#define SFB_CENTRY(ID, DBL, N1, N2, P, TPL1, TPL2, MAXT, MINB, R1, R2)                                      \
    ClusterEntry{ID, DBL, N1, N2, P, TPL1, TPL2, MAXT, MINB, {SFB_EXPAND R1}, {SFB_EXPAND R2}, count_args(SFB_EXPAND R1), \
                 count_args(SFB_EXPAND R2)},
#define SFB_EXPAND(...) __VA_ARGS__
const ClusterEntry kCluster[] = {SFB_CLUSTER_CATALOG(SFB_CENTRY)};
#undef SFB_CENTRY
#undef SFB_EXPAND

const ClusterEntry* find_cluster(bool dbl, int64_t n, int prefer_p) {
    const ClusterEntry* first = nullptr;
    for (const ClusterEntry& e : kCluster) {
        if (e.dbl != (dbl ? 1 : 0) || static_cast<int64_t>(e.n1) * e.n2 != n) continue;
        if (!first) first = &e;
        if (prefer_p == 0 || e.p == prefer_p) return &e;
    }
    return first;
}

#define SFB_PENTRY(ID, DBL, N, TPL, MAXT, ...) PipedEntry{ID, DBL, N, TPL, MAXT, {__VA_ARGS__}, count_args(__VA_ARGS__)},
const PipedEntry kPiped[] = {SFB_PIPED_CATALOG(SFB_PENTRY)};
#undef SFB_PENTRY

const PipedEntry* find_piped(bool dbl, int n) {
    for (const PipedEntry& e : kPiped)
        if (e.dbl == (dbl ? 1 : 0) && e.n == n) return &e;
    return nullptr;
}

#define SFB_TENTRY(ID, R, S, L, COLS, G) \
    TcEntry{ID, R, S, L, COLS, TcShape<R, S, L, G>::N, TcShape<R, S, L, G>::THREADS, int64_t(TcShape<R, S, L, G>::SMEM)},
const TcEntry kTc[] = {SFB_TC_CATALOG(SFB_TENTRY)};
#undef SFB_TENTRY

#define SFB_BENTRY(ID, DBL, KIND, N, TPL, W, MAXT, ...) \
    BlueEntry{ID, DBL, KIND, N, TPL, W, MAXT, {__VA_ARGS__}, count_args(__VA_ARGS__)},
const BlueEntry kBlue[] = {SFB_BLUESTEIN_CATALOG(SFB_BENTRY)};
#undef SFB_BENTRY

const BlueEntry* blue_entries(int* count) {
    *count = static_cast<int>(sizeof(kBlue) / sizeof(kBlue[0]));
    return kBlue;
}

const TcEntry* find_tc(int n, bool cols) {
    for (const TcEntry& e : kTc)
        if (e.n == n && (e.cols != 0) == cols) return &e;
    return nullptr;
}

bool has_fused4(bool dbl, int col_id, int row_id) {
    struct Pair { int dbl, col, row; };
    static const Pair pairs[] = {
#define SFB_X(ID, DBL, N1, TPL1, W1, COL, N2, TPL2, W2, ROW, THREADS, MINB, PERSIST, RC, RR) {DBL, COL, ROW},
        SFB_FUSED4_CATALOG(SFB_X)
#undef SFB_X
    };
    for (const Pair& q : pairs)
        if (q.dbl == (dbl ? 1 : 0) && q.col == col_id && q.row == row_id) return true;
    return false;
}

const FixedEntry* find_fixed(bool dbl, int mode, int n, int feat) {
    for (const FixedEntry& e : kFixed)
        if (e.dbl == (dbl ? 1 : 0) && e.modec == (mode == kModeC ? 1 : 0) && e.n == n && e.feat == feat) return &e;
    return nullptr;
}

// Runtime-length passes whose layout the contiguous kernel (lean_kernel.cuh) covers: whole
// contiguous lines, or the column / row pass of a contiguous four-step, with no table,
// padding or second FFT, at least two stages in the radix order 16, 8, 4, 2, 3, 5, 7 and a
// power-of-two tile width. Values of lean_feat: 0 plain, 1 four-step twiddle.
// Lean passes with 16 values per thread run each (3, 5) pair of stages as one prime-factor
// radix-15 stage: a radix-3, -5 or -15 stage all need n / 15 threads per line at 16 values a
// thread, so the tile shape is unchanged and a shared-memory round trip and a barrier go.
// Returns the new radix sequence, or an empty one when nothing changes.
static std::vector<int> lean_radix15(const PassSpec& ps) {
    const StageSeq& f = ps.p.fft1;
    if (ps.kc.maxv < 16) return {};
    int n3 = 0, n5 = 0;
    for (int s = 0; s < f.nstages; ++s) {
        n3 += f.radix[s] == 3;
        n5 += f.radix[s] == 5;
    }
    const int k = std::min(n3, n5);
    if (k == 0) return {};
    std::vector<int> r;
    for (int s = 0; s < f.nstages; ++s)
        if (f.radix[s] != 3 && f.radix[s] != 5 && f.radix[s] != 7) r.push_back(f.radix[s]);
    for (int i = 0; i < k; ++i) r.push_back(15);
    for (int i = k; i < n3; ++i) r.push_back(3);
    for (int i = k; i < n5; ++i) r.push_back(5);
    for (int s = 0; s < f.nstages; ++s)
        if (f.radix[s] == 7) r.push_back(7);
    // the lean kernel runs at least two stages (a first from and a last to global memory)
    if (r.size() < 2 || threads_per_line(static_cast<int>(ps.p.n), r, ps.kc.maxv) != ps.p.tpl) return {};
    return r;
}

static void mark_lean(PassSpec& ps, int64_t cs) {
    const PassParams& p = ps.p;
    if (ps.fixed_id >= 0 || ps.cluster_id >= 0 || ps.piped_id >= 0 || ps.tc_id >= 0 || ps.blue_id >= 0 || ps.rader ||
        ps.cluster_pipe || ps.tw_base)
        return;
    if (!lean_variant_exists(cs == 16, ps.kc.maxv, ps.kc.maxt)) return;
    if (p.fft2.nstages > 0 || p.fft1.nstages < 2 || ps.tables.premul >= 0 || ps.tables.postmul >= 0 ||
        ps.tables.pointwise >= 0 || ps.tables.perm_in >= 0 || ps.tables.perm_out >= 0)
        return;
    if (p.in.d != 1 || p.out.d != 1 || p.flip_in || p.flip_out || p.w < 1 || (p.w & (p.w - 1)) != 0) return;
    static const int order[] = {16, 8, 4, 2, 15, 3, 5, 7};
    int pos = 0;
    for (int s = 0; s < p.fft1.nstages; ++s) {
        while (pos < 8 && order[pos] != p.fft1.radix[s]) ++pos;
        if (pos == 8) return;  // a radix outside the order, or out of order
    }
    const int64_t n = p.n;
    if (p.mode == kModeK && !p.store_via_smem && p.tw4_sign == 0 && p.sel_mode == kSelNone && p.g_k == 1 &&
        p.in.ks == 1 && p.out.ks == 1 && p.in_len >= n && p.out_len >= n &&
        p.pad_shift == pad_shift_for(cs == 16)) {  // the lean kernel's compile-time row padding
        ps.lean = true;
        ps.lean_feat = 0;
    } else if (p.mode == kModeC && !p.store_via_smem && p.tw4_sign != 0 && p.sel_mode == kSelCol &&
               p.in.cs == 1 && p.out.cs == 1 && p.g_k == p.n_cols && p.in_len >= n * p.g_k && p.out_len >= n * p.g_k &&
               n * p.g_k <= (int64_t(1) << 30)) {
        ps.lean = true;
        ps.lean_feat = 1;
    } else if (p.mode == kModeK && p.store_via_smem && p.tw4_sign == 0 && p.sel_mode == kSelNone && p.g_k == 1 &&
               p.in.ks == 1 && p.out.cs == 1 && p.in_len >= n && p.out_len >= n) {
        // The row pass of a contiguous four-step as a column-tile pass: lanes walk the tile's w
        // adjacent rows (loads are runs of 64 / 128 bytes per row, stores runs of w consecutive
        // output columns), so neither the padded row layout nor a transposed-store phase is
        // needed and every shared-memory address steps linearly.
        PassParams& q = ps.p;
        q.mode = kModeC;
        q.store_via_smem = 0;
        ps.smem_bytes = static_cast<int64_t>(q.w) * q.n * cs;
        ps.lean = true;
        ps.lean_feat = 0;
    }
}

PlanSpec make_plan(const PlanRequest& req) {
    if (req.direction != -1 && req.direction != 1) throw std::invalid_argument("Invalid FFT direction");
    if (req.normalization < 0 || req.normalization > 3) throw std::invalid_argument("Invalid normalization");
    PlanSpec plan;
    plan.req = req;
    plan.elements = checked_element_count(req.shape, req.batch);
    plan.transform_size = 1;
    for (size_t ax = 0; ax < req.shape.size(); ++ax)
        if (!((req.skip_axes >> ax) & 1u)) plan.transform_size *= req.shape[ax];
    plan.scale = normalization_scale(req.normalization, req.direction, plan.transform_size);
    if (plan.elements > (uint64_t(1) << 40)) throw std::invalid_argument("FFT too large for one device");
    Builder b{plan, req, req.dbl ? 16 : 8, req.smem_limit > 0 ? req.smem_limit : kSmemDefault, {}};
    Buf cur = Buf::Input;
    const int rank = static_cast<int>(req.shape.size());
    const int64_t E = static_cast<int64_t>(plan.elements);
    for (int ax = rank - 1; ax >= 0; --ax) {
        const int64_t L = static_cast<int64_t>(req.shape[ax]);
        if (L == 1 || ((req.skip_axes >> ax) & 1u)) continue;
        int64_t s = 1;
        for (int j = ax + 1; j < rank; ++j) s *= static_cast<int64_t>(req.shape[j]);
        b.axis(ax, L, s, E / (L * s), cur);
    }
    if (plan.passes.empty()) b.copy_pass(cur);
    plan.passes.back().p.scale = plan.scale;
    for (auto& ps : plan.passes) {
        mark_lean(ps, req.dbl ? 16 : 8);
        if (!ps.lean) continue;
        const std::vector<int> r = lean_radix15(ps);
        if (!r.empty()) ps.p.fft1 = b.make_seq(static_cast<int>(ps.p.n), r, ps.kc.maxv, &ps.tables.tw1);
    }
    // The batch is the outermost index of every pass: the pass's outer count when it has
    // one (n_outer > 1 or strided columns), else its line count.
    for (auto& ps : plan.passes) {
        const bool outer = ps.p.n_outer > 1 || (ps.p.n_outer == 1 && ps.p.mode == kModeC && req.batch == 1);
        ps.batch_dim = outer ? 0 : 1;
        const int64_t v = ps.batch_dim == 0 ? ps.p.n_outer : ps.p.n_cols;
        if (v % static_cast<int64_t>(req.batch) != 0) ps.batch_dim = -1;  // cannot rescale
    }
    return plan;
}

std::string describe_plan(const PlanSpec& plan) {
    std::ostringstream os;
    os << "{\"elements\":" << plan.elements << ",\"scratch_elements\":" << plan.scratch_elements
       << ",\"tuning\":" << (plan.tuning.empty() ? std::string("null") : plan.tuning)
       << ",\"scale\":" << plan.scale << ",\"passes\":[";
    for (size_t i = 0; i < plan.passes.size(); ++i) {
        const PassSpec& ps = plan.passes[i];
        const PassParams& p = ps.p;
        if (i) os << ",";
        os << "{\"kind\":\"" << ps.kind << "\",\"axis\":" << ps.axis << ",\"n\":" << p.n << ",\"radices\":[";
        for (int s = 0; s < p.fft1.nstages; ++s) os << (s ? "," : "") << p.fft1.radix[s];
        os << "],\"two_ffts\":" << (p.fft2.nstages > 0 ? "true" : "false") << ",\"mode\":\""
           << (p.mode == kModeK ? "k" : "c") << "\",\"tpl\":" << p.tpl << ",\"w\":" << p.w
           << ",\"threads\":" << ps.threads << ",\"smem\":" << ps.smem_bytes << ",\"tiles\":" << p.tiles
           << ",\"maxv\":" << ps.kc.maxv << ",\"maxt\":" << ps.kc.maxt << ",\"src\":" << int(ps.src)
           << ",\"dst\":" << int(ps.dst) << ",\"bytes\":" << ps.bytes_moved
           << ",\"store_via_smem\":" << p.store_via_smem << ",\"fixed_id\":" << ps.fixed_id
           << ",\"piped_id\":" << ps.piped_id << ",\"tc_id\":" << ps.tc_id << ",\"blue_id\":" << ps.blue_id << ",\"tma\":" << (ps.tma ? 1 : 0) << ",\"cluster_id\":" << ps.cluster_id << ",\"cluster_pipe\":" << (ps.cluster_pipe ? 1 : 0) << ",\"cluster\":[" << ps.cl_n1 << "," << ps.cl_n2 << ","
           << ps.cl_p << "],\"rader\":" << (ps.rader ? 1 : 0) << ",\"lean\":" << (ps.lean ? 1 : 0) << "}";
    }
    os << "]}";
    return os.str();
}

}  // namespace sfb
