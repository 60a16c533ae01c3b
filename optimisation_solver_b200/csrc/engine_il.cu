// engine_il.cu -- host side of the batch-interleaved layout of a session:
// the CSR copies of the shared matrix in internal order, the interleaved
// buffers, and the launches of the interleaved trial kernels and of the
// transposes around the per-instance checks.
#include "engine.hpp"

#include <algorithm>
#include <utility>

namespace pdlpgpu {

namespace {

// Line ranges of `ctas` CTAs with about equal work, a line weighing its
// entries plus a fixed cost of four.
std::vector<int32_t> balanced_ranges(const std::vector<int64_t>& ptr, int32_t lines, int ctas) {
    std::vector<int32_t> r(static_cast<size_t>(ctas) + 1, 0);
    const double total = static_cast<double>(ptr[static_cast<size_t>(lines)]) + 4.0 * lines;
    int32_t line = 0;
    for (int c = 1; c < ctas; ++c) {
        const double target = total * c / ctas;
        while (line < lines && static_cast<double>(ptr[static_cast<size_t>(line)]) + 4.0 * line < target) ++line;
        r[static_cast<size_t>(c)] = line;
    }
    r[static_cast<size_t>(ctas)] = lines;
    return r;
}

// Tiles of every CTA's line range (tiles never cross a CTA boundary); fills
// `cta_tiles` with the tile range of each CTA.
int32_t line_segments(int64_t len) {
    return static_cast<int32_t>((len + kIlSegEntries - 1) / kIlSegEntries);
}

// With `segmented`, a staged tile also holds at most kIlTileSegs row segments
// (a row with more forms an unstaged tile of its own).
std::vector<IlTile> make_tiles(const std::vector<int64_t>& ptr, const std::vector<int32_t>& cta_lines,
                               std::vector<int32_t>& cta_tiles, bool segmented) {
    std::vector<IlTile> tiles;
    const size_t ctas = cta_lines.size() - 1;
    cta_tiles.assign(ctas + 1, 0);
    for (size_t c = 0; c < ctas; ++c) {
        cta_tiles[c] = static_cast<int32_t>(tiles.size());
        int32_t i = cta_lines[c];
        const int32_t end = cta_lines[c + 1];
        while (i < end) {
            IlTile t{};
            t.line0 = i;
            t.e0 = ptr[static_cast<size_t>(i)];
            const int64_t len = ptr[static_cast<size_t>(i) + 1] - t.e0;
            if (len > kIlTileEntries || (segmented && line_segments(len) > kIlTileSegs)) {
                t.lines = 1;
                t.entries = static_cast<int32_t>(std::min<int64_t>(ptr[static_cast<size_t>(i) + 1] - t.e0, INT32_MAX));
                t.staged = 0;
                ++i;
            } else {
                int32_t segs = 0;
                while (i < end && i - t.line0 < kIlTileLines &&
                       ptr[static_cast<size_t>(i) + 1] - t.e0 <= kIlTileEntries) {
                    const int64_t li = ptr[static_cast<size_t>(i) + 1] - ptr[static_cast<size_t>(i)];
                    if (segmented && (line_segments(li) > kIlTileSegs || segs + line_segments(li) > kIlTileSegs))
                        break;
                    segs += line_segments(li);
                    ++i;
                }
                t.lines = i - t.line0;
                t.entries = static_cast<int32_t>(ptr[static_cast<size_t>(i)] - t.e0);
                t.staged = 1;
            }
            tiles.push_back(t);
        }
    }
    cta_tiles[ctas] = static_cast<int32_t>(tiles.size());
    return tiles;
}

}  // namespace

int Engine::chunk_slots() const {
    const int slack = spec_.ext.chunk_slack > 0 ? spec_.ext.chunk_slack : 4;
    int slots = std::max(1, std::min(spec_.opt.termination_check_frequency + slack, 1024));
    // Interleaved trials alternate their read buffer with the slot; an even
    // count makes every chunk start reading buffer 0.
    if (il_ && (slots & 1)) ++slots;
    return slots;
}

int Engine::check_stage_launches(bool il_sync) const {
    return (mixed_ ? 8 : 5) + (il_sync && il_ ? 2 : 0) + (dopt_.ndg_restarts ? 1 : 0);
}

template <class T>
bool Engine::il_build(Interleaved<T>& il, const Work<T>& w) {
    const MatrixLayout& L = layouts_[0];
    const int32_t m = L.m, n = L.n;
    il.m = m;
    il.n = n;
    il.count = count_;
    // Instances per lane: the widest load (16 bytes at most) that leaves no
    // group more than half empty.
    const int vmax = sizeof(T) == 4 ? 4 : 2;
    il.vl = 1;
    while (il.vl < vmax && count_ >= 32 * il.vl * 2) il.vl *= 2;
    const int want = spec_.ext.lane_instances;
    if (want == 1 || want == 2 || (want == 4 && vmax == 4)) il.vl = want;
    il.gsize = 32 * il.vl;
    il.bp = (count_ + il.gsize - 1) / il.gsize * il.gsize;
    il.groups = il.bp / il.gsize;

    // The shared matrix in internal order: A by rows (entries by internal
    // column), A^T by columns (entries by internal row).
    std::vector<int32_t> inv_col(static_cast<size_t>(n));
    for (int32_t q = 0; q < n; ++q) inv_col[static_cast<size_t>(L.col_perm[static_cast<size_t>(q)])] = q;
    const int64_t nnz = csr0_.nnz();
    std::vector<int64_t> ap(static_cast<size_t>(m) + 1, 0), tp(static_cast<size_t>(n) + 1, 0);
    std::vector<int32_t> ai(static_cast<size_t>(nnz)), ti(static_cast<size_t>(nnz));
    std::vector<double> av(static_cast<size_t>(nnz)), tv(static_cast<size_t>(nnz));
    std::vector<std::pair<int32_t, double>> row;
    int64_t k = 0;
    for (int32_t r = 0; r < m; ++r) {
        const int32_t o = L.row_perm[static_cast<size_t>(r)];
        row.clear();
        for (int64_t q = csr0_.start[static_cast<size_t>(o)]; q < csr0_.start[static_cast<size_t>(o) + 1]; ++q)
            row.emplace_back(inv_col[static_cast<size_t>(csr0_.index[static_cast<size_t>(q)])],
                             csr0_.value[static_cast<size_t>(q)]);
        std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (const auto& e : row) {
            ai[static_cast<size_t>(k)] = e.first;
            av[static_cast<size_t>(k)] = e.second;
            ++tp[static_cast<size_t>(e.first) + 1];
            ++k;
        }
        ap[static_cast<size_t>(r) + 1] = k;
    }
    for (int32_t q = 0; q < n; ++q) tp[static_cast<size_t>(q) + 1] += tp[static_cast<size_t>(q)];
    {
        std::vector<int64_t> fill(tp.begin(), tp.end() - 1);
        for (int32_t r = 0; r < m; ++r)
            for (int64_t q = ap[static_cast<size_t>(r)]; q < ap[static_cast<size_t>(r) + 1]; ++q) {
                const int64_t d = fill[static_cast<size_t>(ai[static_cast<size_t>(q)])]++;
                ti[static_cast<size_t>(d)] = r;
                tv[static_cast<size_t>(d)] = av[static_cast<size_t>(q)];
            }
    }
    // One wave: as many CTAs over all groups as the multiprocessors hold at
    // once, at least eight lines (one per warp) each.
    const int row_target = std::max(1, sms_ * il_blocks_per_sm<T>(il.vl, true) / il.groups);
    const int col_target = std::max(1, sms_ * il_blocks_per_sm<T>(il.vl, false) / il.groups);
    il.row_ctas = std::max(1, std::min(row_target, (m + 7) / 8));
    il.col_ctas = std::max(1, std::min(col_target, (n + 7) / 8));
    std::vector<int32_t> a_cta, at_cta;
    const std::vector<IlTile> a_tiles = make_tiles(ap, balanced_ranges(ap, m, il.row_ctas), a_cta, true);
    const std::vector<IlTile> at_tiles = make_tiles(tp, balanced_ranges(tp, n, il.col_ctas), at_cta, false);
    std::vector<int32_t> lseg(static_cast<size_t>(m) + 1, 0);
    std::vector<int64_t> segstart;
    for (int32_t r = 0; r < m; ++r) {
        for (int64_t q = ap[static_cast<size_t>(r)]; q < ap[static_cast<size_t>(r) + 1]; q += kIlSegEntries)
            segstart.push_back(q);
        lseg[static_cast<size_t>(r) + 1] = static_cast<int32_t>(segstart.size());
    }
    segstart.push_back(ap[static_cast<size_t>(m)]);

    auto dalloc = [&](auto*& p, size_t count) {
        void* q = nullptr;
        if (!check(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(*p)), "cudaMalloc")) return false;
        extra_.push_back(q);
        p = static_cast<std::remove_reference_t<decltype(p)>>(q);
        return true;
    };
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return bytes == 0 || check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), "upload");
    };
    int64_t *d_ap = nullptr, *d_tp = nullptr;
    int32_t *d_ai = nullptr, *d_ti = nullptr, *d_acta = nullptr, *d_atcta = nullptr;
    IlTile *d_atiles = nullptr, *d_attiles = nullptr;
    int32_t* d_lseg = nullptr;
    int64_t* d_segstart = nullptr;
    double *d_av = nullptr, *d_tv = nullptr;
    T *d_aval = nullptr, *d_tval = nullptr;
    const size_t nb = static_cast<size_t>(n) * il.bp, mb = static_cast<size_t>(m) * il.bp;
    bool ok = dalloc(d_ap, ap.size()) && dalloc(d_tp, tp.size()) && dalloc(d_ai, ai.size()) &&
              dalloc(d_ti, ti.size()) && dalloc(d_av, av.size()) && dalloc(d_tv, tv.size()) &&
              dalloc(d_aval, av.size()) && dalloc(d_tval, tv.size()) && dalloc(d_acta, a_cta.size()) &&
              dalloc(d_atcta, at_cta.size()) && dalloc(d_atiles, a_tiles.size()) &&
              dalloc(d_attiles, at_tiles.size()) && dalloc(d_lseg, lseg.size()) &&
              dalloc(d_segstart, segstart.size());
    for (int b = 0; ok && b < 2; ++b)
        ok = dalloc(il.X[b], nb) && dalloc(il.Y[b], mb) && dalloc(il.AX[b], mb);
    ok = ok && dalloc(il.avg_x, nb) && dalloc(il.avg_y, mb);
    for (int v = 0; ok && v < kIlVecs; ++v) {
        const bool cols = v == kIlC || v == kIlXl || v == kIlXu;
        ok = dalloc(il.own[v], cols ? nb : mb) && dalloc(il.fam[v], static_cast<size_t>(cols ? n : m));
    }
    il.col_batches = (il.col_ctas + kIlBatch - 1) / kIlBatch;
    il.row_batches = (il.row_ctas + kIlBatch - 1) / kIlBatch;
    const size_t G = static_cast<size_t>(il.gsize), ng = static_cast<size_t>(il.groups);
    const size_t cd = ng * (il.row_batches + 1);
    ok = ok && dalloc(il.part_primal, ng * il.col_ctas * G) && dalloc(il.part2_primal, ng * il.col_batches * G) &&
         dalloc(il.part_dual, ng * il.row_ctas * 2 * G) && dalloc(il.part2_dual, ng * il.row_batches * 2 * G) &&
         dalloc(il.cnt_dual, cd);
    if (!ok) return false;
    ok = up(d_ap, ap.data(), ap.size() * 8) && up(d_tp, tp.data(), tp.size() * 8) &&
         up(d_ai, ai.data(), ai.size() * 4) && up(d_ti, ti.data(), ti.size() * 4) &&
         up(d_av, av.data(), av.size() * 8) && up(d_tv, tv.data(), tv.size() * 8) &&
         up(d_acta, a_cta.data(), a_cta.size() * 4) && up(d_atcta, at_cta.data(), at_cta.size() * 4) &&
         up(d_atiles, a_tiles.data(), a_tiles.size() * sizeof(IlTile)) &&
         up(d_attiles, at_tiles.data(), at_tiles.size() * sizeof(IlTile)) &&
         up(d_lseg, lseg.data(), lseg.size() * 4) && up(d_segstart, segstart.data(), segstart.size() * 8);
    for (int b = 0; ok && b < 2; ++b)
        ok = check(cudaMemsetAsync(il.X[b], 0, nb * sizeof(T), stream_), "memset") &&
             check(cudaMemsetAsync(il.Y[b], 0, mb * sizeof(T), stream_), "memset") &&
             check(cudaMemsetAsync(il.AX[b], 0, mb * sizeof(T), stream_), "memset");
    ok = ok && check(cudaMemsetAsync(il.avg_x, 0, nb * sizeof(T), stream_), "memset") &&
         check(cudaMemsetAsync(il.avg_y, 0, mb * sizeof(T), stream_), "memset") &&
         check(cudaMemsetAsync(il.cnt_dual, 0, cd * 4, stream_), "memset");
    if (!ok) return false;
    il.a_ptr = d_ap;
    il.a_idx = d_ai;
    il.a_val = d_aval;
    il.at_ptr = d_tp;
    il.at_idx = d_ti;
    il.at_val = d_tval;
    il.a_cta = d_acta;
    il.at_cta = d_atcta;
    il.a_tiles = d_atiles;
    il.at_tiles = d_attiles;
    il.a_lseg = d_lseg;
    il.a_segstart = d_segstart;
    // Scales and preconditioner are functions of A: instance 0's copies serve
    // every instance.
    launch_il_scale<T>(d_ap, d_ai, d_av, d_aval, g_.rs, g_.cs, m, stream_);
    launch_il_scale<T>(d_tp, d_ti, d_tv, d_tval, g_.cs, g_.rs, n, stream_);
    il.tau = w.tau;
    il.itau = w.itau;
    il.sigma = w.sigma;
    il.isigma = w.isigma;
    launch_il_family<T>(il, fam_, g_.rs, g_.cs, stream_);
    il_set_family((1 << kIlVecs) - 1);
    return check(cudaGetLastError(), "interleaved setup") && check(cudaStreamSynchronize(stream_), "interleaved setup");
}

void Engine::il_set_family(int32_t family) {
    il_family_ = family;
    auto set = [&](auto& il) {
        il.family = family;
        for (int k = 0; k < kIlVecs; ++k) il.vec[k] = ((family >> k) & 1) ? il.fam[k] : il.own[k];
    };
    set(il32_);
    set(il64_);
}

namespace {

template <class T>
void add_pair(IlMove<T>& mv, T* p0, T* p1, T* i0, T* i1, int32_t lines, int by_parity, int by_ibuf) {
    IlPair<T>& P = mv.pair[mv.pairs++];
    P.planar[0] = p0;
    P.planar[1] = p1;
    P.il[0] = i0;
    P.il[1] = i1;
    P.lines = lines;
    P.by_parity = by_parity;
    P.by_ibuf = by_ibuf;
    P.tile0 = mv.tiles;
    mv.tiles += (lines + 31) / 32;
}

}  // namespace

template <class T>
IlMove<T> Engine::il_iterates(const Interleaved<T>& il, const Work<T>& w, bool to_planar, int select,
                              const int32_t* mask) const {
    IlMove<T> mv{};
    const int by_ibuf = to_planar ? 1 : 0;   // inward moves land in buffer 0
    add_pair<T>(mv, w.X[0], w.X[1], il.X[0], il.X[1], il.n, 1, by_ibuf);
    add_pair<T>(mv, w.avg_x, w.avg_x, il.avg_x, il.avg_x, il.n, 0, 0);
    add_pair<T>(mv, w.Y[0], w.Y[1], il.Y[0], il.Y[1], il.m, 1, by_ibuf);
    add_pair<T>(mv, w.AX[0], w.AX[1], il.AX[0], il.AX[1], il.m, 1, by_ibuf);
    add_pair<T>(mv, w.avg_y, w.avg_y, il.avg_y, il.avg_y, il.m, 0, 0);
    mv.to_planar = to_planar ? 1 : 0;
    mv.select = select;
    mv.reset_ibuf = to_planar ? 0 : 1;
    mv.count = il.count;
    mv.bp = il.bp;
    mv.ctl = g_.ctl;
    mv.mask = mask;
    return mv;
}

template <class T>
IlMove<T> Engine::il_statics(const Interleaved<T>& il, const Work<T>& w, int select,
                             const int32_t* mask) const {
    IlMove<T> mv{};
    T* planar[kIlVecs] = {w.c, w.rl, w.ru, w.xl, w.xu};
    for (int k = 0; k < kIlVecs; ++k) {
        if ((il.family >> k) & 1) continue;
        const bool cols = k == kIlC || k == kIlXl || k == kIlXu;
        add_pair<T>(mv, planar[k], planar[k], il.own[k], il.own[k], cols ? il.n : il.m, 0, 0);
    }
    mv.to_planar = 0;
    mv.select = select;
    mv.reset_ibuf = 0;
    mv.count = il.count;
    mv.bp = il.bp;
    mv.ctl = g_.ctl;
    mv.mask = mask;
    return mv;
}

void Engine::il_move_iterates(bool to_planar, int select, const int32_t* mask) {
    if (mixed_) launch_il_move<float>(il_iterates(il32_, w32_, to_planar, select, mask), il32_.bp / 32, stream_);
    else launch_il_move<double>(il_iterates(il64_, w64_, to_planar, select, mask), il64_.bp / 32, stream_);
}

void Engine::il_move_statics(int select, const int32_t* mask) {
    if (mixed_) launch_il_move<float>(il_statics(il32_, w32_, select, mask), il32_.bp / 32, stream_);
    else launch_il_move<double>(il_statics(il64_, w64_, select, mask), il64_.bp / 32, stream_);
}

template bool Engine::il_build<float>(Interleaved<float>&, const Work<float>&);
template bool Engine::il_build<double>(Interleaved<double>&, const Work<double>&);

}  // namespace pdlpgpu
