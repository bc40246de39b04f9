// Host-only check of the shared-memory row strides of the line tiles
// (tile_stride, sns_fft_core.cuh): for every line length and run width that
// the kernels use, the 16 lanes of each half-warp touch 16 distinct 8-byte
// slots (modulo 16) in every access a line FFT makes -- the natural-order
// loads and stores (position j + TPL e) and the stage stores of the Stockham
// stages (position (jb / Ns) Ns R + jb % Ns + r Ns, jb = j + m TPL).  The lane
// layout is that of the tiles: lane t = w + W (j + TPL g), line w + W g.
// Prints the number of conflicting accesses and exits non-zero if any.
#include <cstdio>

#include "sns_fft_core.cuh"

using namespace sns;

template <int L>
int check() {
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL;
  int bad = 0;
  for (int W = 1; W <= 16; W *= 2) {
    const int RS = tile_stride(L, W);
    const int lanes = 32;
    auto slot_of = [&](int t, int pos) {
      const int w = t % W, s = t / W, j = s % TPL, g = s / TPL;
      const int li = w + W * g;
      (void)j;
      return (li * RS + pad_pos(pos)) & 15;
    };
    auto jof = [&](int t) { return (t / W) % TPL; };
    // natural-order accesses
    for (int e = 0; e < E; e++)
      for (int h = 0; h < 2; h++) {
        int used[16] = {0};
        for (int t = 16 * h; t < 16 * h + 16 && t < lanes; t++) used[slot_of(t, jof(t) + TPL * e)]++;
        for (int q = 0; q < 16; q++) bad += used[q] > 1;
      }
    // stage stores
    int Ns = 1;
    for (int st = 0; st + 1 < P::NSTAGE; st++) {
      const int R = P::radix(st);
      for (int m = 0; m < E / R; m++)
        for (int r = 0; r < R; r++)
          for (int h = 0; h < 2; h++) {
            int used[16] = {0};
            for (int t = 16 * h; t < 16 * h + 16; t++) {
              const int jb = jof(t) + m * TPL;
              used[slot_of(t, (jb / Ns) * Ns * R + jb % Ns + r * Ns)]++;
            }
            for (int q = 0; q < 16; q++) bad += used[q] > 1;
          }
      Ns *= R;
    }
  }
  printf("L=%d conflicting half-warp accesses: %d\n", L, bad);
  return bad;
}

int main() {
  int bad = check<16>() + check<32>() + check<64>() + check<128>() + check<256>() + check<512>();
  return bad ? 1 : 0;
}
