// Host-only check of the shared-memory row strides of the line tiles
// (tile_stride, sns_fft_core.cuh): for every line length and run width that
// the kernels use, the P = 128 / esz lanes of each access group (a half-warp
// of 8-byte complex64 elements, a quarter-warp of 16-byte complex128 ones)
// touch P distinct element slots (modulo P) in every access a line FFT makes:
// the natural-order loads and stores (position j + TPL e) and the stage stores of the Stockham
// stages (position (jb / Ns) Ns R + jb % Ns + r Ns, jb = j + m TPL).  The lane
// layout is that of the tiles: lane t = w + W (j + TPL g), line w + W g.
// Prints the number of conflicting accesses and exits non-zero if any.
#include <cstdio>

#include "sns_fft_core.cuh"

using namespace sns;

template <int L, int ESZ>
int check() {
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL;
  constexpr int G = 128 / ESZ;  // lanes per access group
  int bad = 0;
  for (int W = 1; W <= 16; W *= 2) {
    const int RS = tile_stride(L, W, ESZ);
    auto slot_of = [&](int t, int pos) {
      const int w = t % W, s = t / W, g = s / TPL;
      const int li = w + W * g;
      return (li * RS + pad_pos(pos)) % G;
    };
    auto jof = [&](int t) { return (t / W) % TPL; };
    // natural-order accesses
    for (int e = 0; e < E; e++)
      for (int h = 0; h < 32 / G; h++) {
        int used[16] = {0};
        for (int t = G * h; t < G * h + G; t++) used[slot_of(t, jof(t) + TPL * e)]++;
        for (int q = 0; q < G; q++) bad += used[q] > 1;
      }
    // stage stores
    int Ns = 1;
    for (int st = 0; st + 1 < P::NSTAGE; st++) {
      const int R = P::radix(st);
      for (int m = 0; m < E / R; m++)
        for (int r = 0; r < R; r++)
          for (int h = 0; h < 32 / G; h++) {
            int used[16] = {0};
            for (int t = G * h; t < G * h + G; t++) {
              const int jb = jof(t) + m * TPL;
              used[slot_of(t, (jb / Ns) * Ns * R + jb % Ns + r * Ns)]++;
            }
            for (int q = 0; q < G; q++) bad += used[q] > 1;
          }
      Ns *= R;
    }
  }
  printf("L=%d esz=%d conflicting accesses: %d\n", L, ESZ, bad);
  return bad;
}

template <int ESZ>
int check_all() {
  return check<16, ESZ>() + check<32, ESZ>() + check<64, ESZ>() + check<128, ESZ>() +
         check<256, ESZ>() + check<512, ESZ>();
}

int main() {
  const int bad = check_all<8>() + check_all<16>();
  return bad ? 1 : 0;
}
