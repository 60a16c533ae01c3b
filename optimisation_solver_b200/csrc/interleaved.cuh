// interleaved.cuh -- the batch-interleaved layout of a shared-matrix session.
//
// A session solves B instances that share one constraint matrix. In this
// layout the trial kernels keep every per-instance vector as [line][Bp]
// (Bp = B rounded up to 32): the 32 instances of a "group" sit side by side,
// so one warp processes one row (or column) for 32 instances at once. The
// matrix is read with warp-uniform loads (every lane needs the same entry),
// and every vector access -- the line's own values and each gathered entry --
// is one coalesced 128-byte (FP32) or 256-byte (FP64) access. Per-instance
// scalars (step, weight, averaging fraction) live in registers of the lane.
//
// Vectors that every instance takes from the family (not loaded per
// instance), and the Ruiz/Pock-Chambolle vectors (functions of A alone), are
// stored once as [line] and broadcast.
//
// Committed iterates and their trial successors use two buffers per vector.
// Trial slot s of a captured chunk reads buffer R = s & 1 and writes the
// trial point to W = R ^ 1 for every lane, so the warp's stores stay
// coalesced. An instance whose last trial was rejected (or that idled) has
// its committed point in the other buffer (InstanceCtl::ibuf); its lane
// reads from there and copies the point into R as it goes, so after the trial
// the committed point is in R (rejected) or W (accepted).
//
// The termination checks keep the per-instance SELL-G layout: before a
// check the iterates of the instances at a check are transposed out, after
// it (restarts, polishing entry, refreshed A x) transposed back in.
#pragma once

#include "common.cuh"

#include <cuda_runtime.h>

namespace pdlpgpu {

// A tile: consecutive lines of one CTA whose entries are staged in shared
// memory together (at most kIlTileLines lines and kIlTileEntries entries). A
// line with more entries forms a tile of its own that reads them from global
// memory (staged = 0).
constexpr int kIlTileLines = 64;
constexpr int kIlTileEntries = 1536;
// The dual splits each row into segments of at most kIlSegEntries entries; a
// warp gathers one segment's entries at once and a row adds its segments'
// partial sums in order. A staged row tile holds at most kIlTileSegs
// segments.
constexpr int kIlSegEntries = 8;
constexpr int kIlTileSegs = 32;

struct IlTile {
    int64_t e0;        // first entry
    int32_t line0;     // first line
    int32_t lines;
    int32_t entries;
    int32_t staged;
};

// Problem vectors of the interleaved layout, in this order.
enum : int32_t { kIlC = 0, kIlRl = 1, kIlRu = 2, kIlXl = 3, kIlXu = 4, kIlVecs = 5 };

// CTAs per first-level batch of the per-group reductions.
constexpr int kIlBatch = 16;

template <class T>
struct Interleaved {
    int32_t m, n;            // rows and columns of the shared matrix
    int32_t count;           // instances B
    int32_t vl;              // instances per lane V (1, 2 or 4): one V-wide load per lane
    int32_t gsize;           // instances per group G = 32 V (one warp covers a group)
    int32_t bp;              // B rounded up to G
    int32_t groups;          // bp / G
    int32_t row_ctas, col_ctas;   // CTAs per group of the dual / primal kernel
    int32_t row_batches, col_batches;   // ceil(ctas / kIlBatch)
    // iterates, [line][bp]
    T* X[2];
    T* Y[2];
    T* AX[2];
    T* avg_x;
    T* avg_y;
    // scaled problem vectors: vec[k] points at own[k] ([line][bp]) or at
    // fam[k] ([line]) when bit k of `family` is set
    const T* vec[kIlVecs];
    T* own[kIlVecs];
    T* fam[kIlVecs];
    int32_t family;
    // preconditioner, [line]
    const T* tau;
    const T* itau;
    const T* sigma;
    const T* isigma;
    // scaled matrix in CSR, internal order: A by rows, A^T by columns
    const int64_t* a_ptr;
    const int32_t* a_idx;
    const T* a_val;
    const int64_t* at_ptr;
    const int32_t* at_idx;
    const T* at_val;
    // tiles of each side and the tile ranges of the CTAs ([row_ctas + 1] /
    // [col_ctas + 1]; CTA line ranges are balanced by entries)
    const IlTile* a_tiles;
    const IlTile* at_tiles;
    // row segments: row i's segments are a_lseg[i] .. a_lseg[i + 1] - 1;
    // segment q starts at entry a_segstart[q]
    const int32_t* a_lseg;      // [m + 1]
    const int64_t* a_segstart;  // [segments + 1]
    const int32_t* a_cta;
    const int32_t* at_cta;
    // Per-instance sums, two levels: every CTA writes its partial, the last
    // CTA of each batch of kIlBatch CTAs adds the batch, the last batch adds
    // the batches -- always in index order.
    // The primal kernel only writes its CTA partials; the dual kernel's CTAs
    // add them by batch before their own arrival.
    double* part_primal;     // [groups][col_ctas][G]
    double* part2_primal;    // [groups][col_batches][G]
    double* part_dual;       // [groups][row_ctas][2][G]
    double* part2_dual;      // [groups][row_batches][2][G]
    int32_t* cnt_dual;       // [groups][row_batches + 1] arrival counters
};

// Which instances a transpose moves.
enum : int32_t {
    kIlAll = 0,       // every instance
    kIlMasked = 1,    // slot_mask[b] != 0
    kIlAtCheck = 2,   // stage == check (sets il_sync)
    kIlSynced = 3     // il_sync != 0
};

// One vector pair of a transpose between the per-instance layout
// (planar[b * lines + line]) and the interleaved one (il[line * bp + b]).
template <class T>
struct IlPair {
    T* planar[2];       // [0] or [parity]
    T* il[2];           // [0] or [ibuf]
    int32_t lines;
    int32_t by_parity;  // planar side indexed by the instance's parity
    int32_t by_ibuf;    // interleaved side indexed by the instance's ibuf
    int32_t tile0;      // first tile of this pair in the launch
};

constexpr int kIlMaxPairs = 6;

template <class T>
struct IlMove {
    IlPair<T> pair[kIlMaxPairs];
    int32_t pairs;
    int32_t tiles;          // total 32-line tiles over the pairs
    int32_t to_planar;      // 1: interleaved -> planar, 0: planar -> interleaved
    int32_t select;         // kIl*
    int32_t reset_ibuf;     // planar -> interleaved of the iterates: ibuf = 0
    int32_t count, bp;
    InstanceCtl* ctl;
    const int32_t* mask;
};

// Resident CTAs per multiprocessor of the dual (or primal) trial kernel with
// `vl` instances per lane.
template <class T>
int il_blocks_per_sm(int vl, bool dual);

template <class T>
void launch_il_primal(const Interleaved<T>& il, InstanceCtl* ctl, int measure, int slot,
                      cudaStream_t s);
template <class T>
void launch_il_dual(const Interleaved<T>& il, InstanceCtl* ctl, const DeviceOptions& o,
                    int measure, int slot, cudaStream_t s);
// `groups`: bp / 32 (a transpose tile covers 32 instances).
template <class T>
void launch_il_move(const IlMove<T>& mv, int groups, cudaStream_t s);
// Scaled values of the CSR copies: val[k] = orig[k] * (line_scale[line] * other[idx[k]]).
template <class T>
void launch_il_scale(const int64_t* ptr, const int32_t* idx, const double* orig, T* val,
                     const double* line_scale, const double* other_scale, int32_t lines,
                     cudaStream_t s);
// Family vectors in working coordinates (as k_setup_vectors scales them).
template <class T>
void launch_il_family(const Interleaved<T>& il, const double* const fam[kIlVecs],
                      const double* rs, const double* cs, cudaStream_t s);

}  // namespace pdlpgpu
