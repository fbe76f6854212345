// Device Welsh-Powell coloring of the constraint rows (coloring.py:26-89):
// arguments, scratch layout and launch of the one-CTA coloring pass.
#pragma once
#include "engine.cuh"

namespace xpbd {

constexpr int kColThreads = 1024;
constexpr int kColMaxColors = 128;       // two 64-bit words of used colors per body
constexpr int kColSmemBodies = 4096;     // bitsets and degrees in shared memory up to this many bodies
constexpr int kColSmemRows = 8192;       // staged chunks in shared memory up to this many live rows
// 16 B x 4096 bodies + max(4 B x 4096 + the sort's work area, 16 B x 8192 rows) = 192 KB

struct ColorArgs {
  const int4* ri;       // rows: type, a, b, active
  const int* n_rows;    // live row count (device)
  int n;                // bodies
  int cap;              // row capacity
  int* color;           // [cap]
  int* order;           // [cap] rows sorted by color (stable)
  int* starts;          // [kColMaxColors + 1]
  int* ncolors;         // [1]
  int* status;          // XPBD_ERR_OVERFLOW: more than kColMaxColors colors needed
  uint64_t *k0, *k1;    // [cap] sort keys
  uint32_t *v0, *v1;    // [cap] sort values
  int* deg;             // [n] (global fallback)
  int4* stage;          // [cap] (global fallback when the live rows exceed kColSmemRows)
  ulonglong2* used;     // [n]   (global fallback when n > kColSmemBodies)
};

size_t color_scratch_bytes(int n, int cap);
void color_scratch_carve(ColorArgs& A, void* scratch, int n, int cap);
// Colors the live rows of A on `st` (asynchronous, capturable).
int color_rows_launch(const ColorArgs& A, cudaStream_t st);

}  // namespace xpbd
