// Device-side data model of the shrink-wrap / HIO engine.
//
// One reconstruction ("job") is the state the reference's cudaShrinkWrap keeps
// in dpCurData / dpgPrevious / dpIntensity / dpIsMasked
// (src/imresh/algorithms/cuda/cudaShrinkWrap.cu:203-214), re-laid out for
// fused passes:
//   X    complex64 [H][W]  the iterate between the row and column passes
//                          (row-transformed g after a row pass; column-
//                          projected, column-inverse-transformed after a
//                          column pass)
//   G    complex64 [H][W]  g_prev of the HIO update
//   M    float32   [H][W]  the Fourier modulus (the caller's input)
//   mask uint8     [H][W]  1 = outside the support (the reference's float 1.0)
//   hb   float32   [H][W]  |g'| blurred along rows
//   vb   float32   [H][W]  |g'| blurred along rows and columns
//   out  float32   [H][W]  Re(g') -- the result
// The same layout serves the fixed-support HIO of libs::hybridInputOutput
// (mode 1): the caller's mask, a random initial phase, no blur, an error and
// stop test after every iteration.
// All per-cycle control (sigma weights, threshold, error, stop test) stays on
// the device, so a reconstruction runs without host synchronisation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cuda.h>
#include "fft_dev.cuh"

namespace imr {

constexpr int kMaxTaps = 63;        // Gaussian kernel taps (half width <= 31)
constexpr int kTapStride = 64;      // floats per cycle in the weight table
constexpr int kRowThreads = 256;
constexpr int kRowVpt = 8;          // complex values per thread per pass (rows, runtime length)
constexpr int kColThreads = 256;
constexpr int kColVpt = 8;          // complex values per thread per pass (columns, runtime length)
constexpr int kVbTileX = 32;
constexpr int kVbTileY = 128;
constexpr int kVbThreads = 256;

struct JobState {
    int cycle;          // cycle whose mask is being built by finish/vblur
                        // (mode 1: the iteration whose g' the next row pass makes)
    int hio_cycle;      // cycle whose HIO block is running
    int stop;           // 1: finished; every later launch returns at once
    int cycles_done;    // HIO blocks completed and error-tested (mode 1: iterations)
    float thr;          // support threshold of the running cycle
    unsigned max_bits;  // max of the blurred |g'| (float bits, values >= 0)
    unsigned counter;   // last-block detection (vertical blur pass; mode 1: row pass)
    float last_error;
    int err;            // nonzero: a device-side wait gave up (see tma.cuh)
};

constexpr int kModeShrinkWrap = 0;
constexpr int kModeHio = 1;   // fixed support, random initial phase

struct alignas(64) JobDev {
    CUtensorMap tmX;    // X as W x H 8-byte elements, box (cpc, rows)
    CUtensorMap tmM;    // M as W x H floats, box (cpc, rows)
    CUtensorMap tmXh;   // X as tmX with box (cpc / 2, rows): half tiles of the column pass
    int use_tma_cols;   // 1: column pass reads tiles through tmX / tmM
    int mode;           // kModeShrinkWrap / kModeHio
    int W, H;
    float2 *X;
    float2 *G;
    const float *M;
    // The modulus in column tiles for the pipelined 16-value column pass, or
    // null: tile t (columns t*cpc .. t*cpc + cpc - 1) is a contiguous [H][cpc]
    // block, zero past column W, so a tile arrives by one bulk copy.
    const float *Mt;
    uint8_t *mask;
    float *hb;
    float *vb;
    float *out;
    FftPlanDev prow;    // length W
    FftPlanDev pcol;    // length H
    float beta, cut_auto, cut, target;
    int n_cycles, n_hio;
    const float *weights;   // [(n_cycles + 1) * kTapStride]
    const int *ntaps;       // [n_cycles + 1]
    double *err_part;       // [2 * n_row_tiles]  (sum mask*|g'|, sum mask)
    float *errors;          // [n_cycles] error after each cycle (mode 1: [n_err] per iteration)
    int n_err;              // mode 1: length of errors
    JobState *st;
    int rpc;                // rows per row-pass CTA
    int cpc;                // columns per column-pass CTA
    int n_row_tiles, n_col_tiles, n_vb_tiles, vb_tiles_x;
    unsigned long long wait_ns;   // limit of each bounded copy wait (0: kWaitNs, 0.5 s)
};

// One unit of work: job index and tile (row group / column group) index.
struct WorkItem {
    int job;
    int tile;
};

// A launch's items, in device memory.  items == nullptr: job 0, tiles 0..n-1.
// n_split (items == nullptr, pipelined 16-value column pass only): tiles
// 0..n_split-1 run as two half-width items each, the first halves before all
// other items and the second halves after them (with n_split = n: every tile
// as two halves, on twice as many CTAs).
struct WorkList {
    const WorkItem *items;
    int n;
    int n_split;
};

}  // namespace imr
