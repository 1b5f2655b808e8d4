// CPU emulator of the B200 provider's pass contract -- TEST INFRASTRUCTURE ONLY.
//
// Builds a plan with the product planner (sycl-fft_b200/csrc/planner.cpp) and runs
// every pass on the host in FP64, following the kernel's semantics step by step:
// per tile line, load with zero-padding/pre-multiply/conjugation, the Stockham stage
// sequence with the planner's twiddle tables, the point-wise multiply and second
// FFT, and the store with conjugation, four-step twiddle, post-multiply, scale and
// truncation, the Rader gather, bin-0 term and scatter. Used by tests/ to check plan
// decompositions (four-step, Bluestein, Rader, strided axes) without a GPU. Never used by
// the product library.
#include <complex>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../sycl-fft_b200/csrc/planner.hpp"

using cd = std::complex<double>;
using namespace sfb;

namespace {

int64_t line_base(const LineLayout& L, int64_t o, int64_t c) {
    return (L.d == 1 ? o * L.hi : (o / L.d) * L.hi + (o % L.d) * L.lo) + c * L.cs;
}

// base == true: the table holds, per stage, W_(Ns*R)^jm (size-specialised kernels), and the
// stage twiddle W^(r*jm) is its r-th power; otherwise the full [Ns][R-1] layout at tw_off.
void stockham(std::vector<cd>& x, const StageSeq& S, const std::vector<cd>& tw, int n, bool base = false) {
    std::vector<cd> y(n);
    int64_t boff = 0;
    for (int s = 0; s < S.nstages; ++s) {
        const int R = S.radix[s], Ns = S.ns[s], nr = n / R;
        for (int j = 0; j < nr; ++j) {
            const int jm = j % Ns;
            cd v[16], u[16];
            for (int r = 0; r < R; ++r) {
                v[r] = x[j + r * nr];
                if (r > 0 && Ns > 1) v[r] *= base ? std::pow(tw[boff + jm], r) : tw[S.tw_off[s] + jm * (R - 1) + (r - 1)];
            }
            for (int p = 0; p < R; ++p) {
                cd acc = 0.0;
                for (int q = 0; q < R; ++q) acc += v[q] * cis_neg(int64_t(p) * q, R);
                u[p] = acc;
            }
            const int base = (j - jm) * R + jm;
            for (int r = 0; r < R; ++r) y[base + r * Ns] = u[r];
        }
        x.swap(y);
        boff += Ns;
    }
}

// Cluster pass: columns (length n1, stride n2) with the n1 stage table, four-step twiddle,
// rows (length n2) with the n2 stage table, stored transposed -- per line.
void run_cluster(const PlanSpec& plan, const PassSpec& ps, const cd* src, cd* dst) {
    const PassParams& p = ps.p;
    const int n1 = ps.cl_n1, n2 = ps.cl_n2, N = n1 * n2;
    const auto& hi = plan.tables[ps.tables.tw4_hi];
    const auto& lo = plan.tables[ps.tables.tw4_lo];
    std::vector<cd> line(N), y(N), col(n1), row(n2);
    for (int64_t c = 0; c < p.n_cols; ++c) {
        for (int k = 0; k < N; ++k) {
            line[k] = src[c * p.in.cs + k];
            if (p.conj_in) line[k] = std::conj(line[k]);
        }
        for (int b = 0; b < n2; ++b) {
            for (int a = 0; a < n1; ++a) col[a] = line[int64_t(a) * n2 + b];
            stockham(col, p.fft1, plan.tables[ps.tables.tw1], n1);
            for (int k1 = 0; k1 < n1; ++k1) {
                const int64_t m = int64_t(k1) * b;
                y[int64_t(k1) * n2 + b] = col[k1] * hi[m >> p.tw4_shift] * lo[m & ((int64_t(1) << p.tw4_shift) - 1)];
            }
        }
        for (int k1 = 0; k1 < n1; ++k1) {
            for (int b = 0; b < n2; ++b) row[b] = y[int64_t(k1) * n2 + b];
            stockham(row, p.fft2, plan.tables[ps.tables.tw2], n2);
            for (int k2 = 0; k2 < n2; ++k2) {
                cd v = row[k2];
                if (p.conj_out) v = std::conj(v);
                dst[c * p.out.cs + k1 + int64_t(n1) * k2] = v * p.scale;
            }
        }
    }
}

// The bin-0 term of a Rader convolution pass (kFeatRaderDC): line starts of the axis input
// and output, their pitch, and the scale of the outputs around it.
struct RaderDC {
    const cd* x = nullptr;
    cd* y = nullptr;
    int64_t x_pitch = 0, y_pitch = 0;
    double scale = 1.0;
};

void run_pass(const PlanSpec& plan, const PassSpec& ps, const cd* src, cd* dst, const RaderDC& dc = RaderDC()) {
    if (ps.cluster_id >= 0) {
        run_cluster(plan, ps, src, dst);
        return;
    }
    const PassParams& p = ps.p;
    auto table = [&](int id) -> const std::vector<cd>* { return id < 0 ? nullptr : &plan.tables[id]; };
    const auto* premul = table(ps.tables.premul);
    const auto* pointwise = table(ps.tables.pointwise);
    const auto* postmul = table(ps.tables.postmul);
    const auto* hi = table(ps.tables.tw4_hi);
    const auto* lo = table(ps.tables.tw4_lo);
    auto itable = [&](int id) -> const std::vector<int32_t>* { return id < 0 ? nullptr : &plan.index_tables[id]; };
    const auto* perm_in = itable(ps.tables.perm_in);
    const auto* perm_out = itable(ps.tables.perm_out);
    // Read every tile line first so in-place passes behave like the kernel (a tile is read
    // before it is written, and tiles are disjoint).
    struct Line { int64_t o, c; std::vector<cd> v; };
    std::vector<Line> lines;
    for (int64_t o = 0; o < p.n_outer; ++o) {
        for (int64_t c = 0; c < p.n_cols; ++c) {
            Line L{o, c, std::vector<cd>(p.n)};
            const int64_t sel = p.sel_mode == kSelCol ? c : p.sel_mode == kSelOuterLo ? o % p.sel_d
                                : p.sel_mode == kSelColMod ? c % p.sel_d : 0;
            const int64_t ib = line_base(p.in, o, c);
            for (int k = 0; k < p.n; ++k) {
                const int64_t g = int64_t(k) * p.g_k + sel;
                cd a = 0.0;
                if (g < p.in_len) {
                    // Rader gather: element g of the line is x[perm_in[g]] (from the line start)
                    a = perm_in ? src[ib - sel + (*perm_in)[g]] : src[ib + int64_t(k) * p.in.ks];
                    if (premul) a *= (*premul)[g];
                    if (p.conj_in) a = std::conj(a);
                }
                L.v[k] = a;
            }
            lines.push_back(std::move(L));
        }
    }
    for (auto& L : lines) {
        const int64_t sel = p.sel_mode == kSelCol ? L.c : p.sel_mode == kSelOuterLo ? L.o % p.sel_d
                            : p.sel_mode == kSelColMod ? L.c % p.sel_d : 0;
        stockham(L.v, p.fft1, plan.tables[ps.tables.tw1], p.n, ps.tw_base);
        if (p.fft2.nstages > 0) {
            cd x0 = 0.0;
            if (ps.rader && sel == 0) {
                // bin 0: X[0] = x[0] + sum of the gathered line; x[0] joins bin 0 of the product
                const bool fused = perm_in != nullptr;
                const int64_t line = fused ? L.c : L.c / p.sel_d;
                const cd* xl = fused ? src + line_base(p.in, L.o, L.c) : dc.x + line * dc.x_pitch;
                cd* yl = fused ? dst + line_base(p.out, L.o, L.c) : dc.y + line * dc.y_pitch;
                x0 = xl[0];
                yl[0] = (x0 + L.v[0]) * (fused ? p.scale : dc.scale);
            }
            for (int k = 0; k < p.n; ++k) {
                if (pointwise) L.v[k] *= (*pointwise)[k + sel * p.pw_stride];
                if (k == 0) L.v[0] += x0;
                if (p.conj_mid) L.v[k] = std::conj(L.v[k]);
            }
            stockham(L.v, p.fft2, plan.tables[ps.tables.tw2], p.n, ps.tw_base);
        }
        const int64_t ob = line_base(p.out, L.o, L.c);
        const bool tstore = ps.fixed_id >= 0 && ps.fixed_feat == kFixedTStore;
        for (int k = 0; k < p.n; ++k) {
            const int64_t g = int64_t(k) * p.g_k + sel;
            if (g >= p.out_len) continue;
            cd v = L.v[k];
            if (p.conj_out) v = std::conj(v);
            if (p.tw4_sign != 0) {
                const int64_t m = int64_t(k) * sel;
                cd w = (*hi)[m >> p.tw4_shift] * (*lo)[m & ((int64_t(1) << p.tw4_shift) - 1)];
                if (p.tw4_sign > 0) w = std::conj(w);
                v *= w;
            }
            if (postmul) v *= (*postmul)[g];
            v *= p.scale;
            if (tstore) {
                // size-specialised row pass: flat row l stored transposed
                const int64_t l = L.c, o = l / p.ts_rows;
                dst[o * p.ts_line + (l - o * p.ts_rows) + int64_t(k) * p.ts_rows] = v;
                continue;
            }
            if (perm_out) {
                dst[ob - sel + (*perm_out)[g]] = v;  // Rader scatter
                continue;
            }
            dst[ob + int64_t(k) * p.out.ks] = v;
        }
    }
}

void set_err(char* err, size_t cap, const std::string& m) {
    if (!err || !cap) return;
    size_t n = std::min(cap - 1, m.size());
    std::memcpy(err, m.data(), n);
    err[n] = 0;
}

}  // namespace

// Plan description only (no execution): the planner's choice for a request.
extern "C" int emu_describe(int dbl, int dir, int norm, int in_place, unsigned rank, const uint64_t* shape,
                            uint64_t batch, int force_maxv, int smem_limit, int split_bf16, char* desc,
                            size_t desc_cap, char* err, size_t cap) {
    try {
        PlanRequest req;
        req.dbl = dbl != 0;
        req.direction = dir;
        req.normalization = norm;
        req.in_place = in_place != 0;
        req.shape.assign(shape, shape + rank);
        req.batch = batch;
        req.force_maxv = force_maxv;
        req.smem_limit = smem_limit;
        req.split_bf16 = split_bf16 != 0;
        req.device_spectrum = true;
        const char* rd = std::getenv("SYCLFFT_B200_RADER");
        req.no_rader = rd && std::strcmp(rd, "0") == 0;
        set_err(desc, desc_cap, describe_plan(make_plan(req)));
        return 0;
    } catch (const std::exception& e) {
        set_err(err, cap, e.what());
        return 1;
    }
}

namespace {

int run_request(int dbl, int dir, int norm, int in_place, unsigned rank, const uint64_t* shape, uint64_t batch,
                int force_maxv, int smem_limit, unsigned skip_axes, const double* in, double* out, char* desc,
                size_t desc_cap, char* err, size_t cap) {
    try {
        PlanRequest req;
        req.dbl = dbl != 0;
        req.direction = dir;
        req.normalization = norm;
        req.in_place = in_place != 0;
        req.shape.assign(shape, shape + rank);
        req.batch = batch;
        req.force_maxv = force_maxv;
        req.smem_limit = smem_limit;
        req.skip_axes = skip_axes;
        // the provider's switch for fused four-step routing of lines that fit one block
        const char* fs = std::getenv("SYCLFFT_B200_FUSED4_SINGLE");
        req.fused_single = fs && std::strcmp(fs, "1") == 0;
        // the provider's switch that keeps prime lengths on Bluestein's convolution
        const char* rd = std::getenv("SYCLFFT_B200_RADER");
        req.no_rader = rd && std::strcmp(rd, "0") == 0;
        PlanSpec plan = make_plan(req);
        set_err(desc, desc_cap, describe_plan(plan));
        const int64_t E = static_cast<int64_t>(plan.elements);
        std::vector<cd> input(E), output(E), scratch(plan.scratch_elements);
        for (int64_t i = 0; i < E; ++i) input[i] = cd(in[2 * i], in[2 * i + 1]);
        if (req.in_place) output = input;
        auto buf = [&](Buf b) -> cd* {
            if (b == Buf::Input) return req.in_place ? output.data() : input.data();
            if (b == Buf::Output) return output.data();
            return scratch.data();
        };
        for (size_t i = 0; i < plan.passes.size(); ++i) {
            const PassSpec& ps = plan.passes[i];
            RaderDC dc;
            if (ps.rader_dc) {
                // between the Rader column passes: their line pitches and the outputs' scale
                dc.x = buf(ps.rader_src);
                dc.y = output.data();
                dc.x_pitch = plan.passes[i - 1].p.in.hi;
                dc.y_pitch = plan.passes[i + 1].p.out.hi;
                dc.scale = plan.passes[i + 1].p.scale;
            }
            run_pass(plan, ps, buf(ps.src), buf(ps.dst), dc);
        }
        for (int64_t i = 0; i < E; ++i) {
            out[2 * i] = output[i].real();
            out[2 * i + 1] = output[i].imag();
        }
        return 0;
    } catch (const std::exception& e) {
        set_err(err, cap, e.what());
        return 1;
    }
}

}  // namespace

extern "C" int emu_run(int dbl, int dir, int norm, int in_place, unsigned rank, const uint64_t* shape,
                       uint64_t batch, int force_maxv, int smem_limit, const double* in, double* out,
                       char* desc, size_t desc_cap, char* err, size_t cap) {
    return run_request(dbl, dir, norm, in_place, rank, shape, batch, force_maxv, smem_limit, 0u, in, out, desc,
                       desc_cap, err, cap);
}

// Like emu_run with axes left untransformed (bit ax of skip_axes: PlanRequest::skip_axes).
extern "C" int emu_run_skip(int dbl, int dir, int norm, int in_place, unsigned rank, const uint64_t* shape,
                            uint64_t batch, unsigned skip_axes, const double* in, double* out, char* desc,
                            size_t desc_cap, char* err, size_t cap) {
    return run_request(dbl, dir, norm, in_place, rank, shape, batch, 0, 0, skip_axes, in, out, desc, desc_cap, err,
                       cap);
}

// The generator the planner's Rader tables are built from.
extern "C" uint64_t emu_primitive_root(uint64_t p) { return primitive_root(p); }
