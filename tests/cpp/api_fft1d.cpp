// The FFT1D class (src/FFT1D.H:18-47) on host and device lines: every public
// entry point -- init + transform(ptr, DIR), transform(ptr, N, stride, DIR),
// forward, inverse -- on strided lines of seeded values.  Each case writes
// int64 {case, N, stride, DIR, length} and then the buffer before and after
// the call (interleaved complex doubles) to the output file; the test compares
// the lines with numpy's DFT and checks that the elements between the strided
// positions are untouched.
// Usage: api_fft1d out.bin
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "DataObjects.H"
#include "../../include/spectral_b200.h"

namespace {

std::vector<cdouble> seeded(size_t n, unsigned seed) {
  std::vector<cdouble> v(n);
  unsigned s = seed * 2654435761u + 12345u;
  auto next = [&]() {
    s = s * 1664525u + 1013904223u;
    return (double)(s >> 8) / (double)(1u << 24) * 2.0 - 1.0;
  };
  for (auto& x : v) x = cdouble(next(), next());
  return v;
}

void record(FILE* f, long long kase, long long N, long long stride, long long dir,
            const std::vector<cdouble>& before, const std::vector<cdouble>& after) {
  long long h[5] = {kase, N, stride, dir, (long long)before.size()};
  fwrite(h, sizeof(h), 1, f);
  fwrite(before.data(), sizeof(cdouble), before.size(), f);
  fwrite(after.data(), sizeof(cdouble), after.size(), f);
}

// kind: 0 transform(ptr,N,stride,DIR), 1 forward, 2 inverse, 3 init+transform(ptr,DIR)
void run(FFT1D& fft, int kind, cdouble* p, int N, int stride, int dir) {
  switch (kind) {
    case 0: fft.transform(p, N, stride, dir); break;
    case 1: fft.forward(p, N, stride); break;
    case 2: fft.inverse(p, N, stride); break;
    default:
      fft.init(N, stride, p);
      fft.transform(p, dir);
      break;
  }
}

}  // namespace

int main(int argc, char* argv[]) {
  if (argc < 2) return 2;
  upcxx::init();
  FILE* f = fopen(argv[1], "wb");
  if (!f) return 3;
  struct Case {
    int kind, N, stride, dir;
  };
  const Case cases[] = {{0, 256, 3, -1}, {0, 64, 1, 1},   {1, 512, 2, -1}, {2, 128, 5, 1},
                        {3, 1024, 1, 1}, {3, 32, 7, -1},  {1, 16, 1, -1},  {2, 4096, 1, 1}};
  long long kase = 0;
  for (int on_device = 0; on_device < 2; on_device++) {
    for (const Case& c : cases) {
      const size_t len = (size_t)(c.N - 1) * c.stride + 1 + 3;  // 3 trailing guards
      std::vector<cdouble> before = seeded(len, (unsigned)(kase + 1));
      std::vector<cdouble> after(before);
      FFT1D fft;
      if (on_device) {
        void* d = nullptr;
        if (sns_malloc(&d, len * sizeof(cdouble)) != SNS_OK) return 4;
        sns_memcpy_h2d(d, before.data(), len * sizeof(cdouble), nullptr);
        run(fft, c.kind, static_cast<cdouble*>(d), c.N, c.stride, c.dir);
        sns_memcpy_d2h(after.data(), d, len * sizeof(cdouble), nullptr);
        sns_stream_synchronize(nullptr);
        sns_free(d);
      } else {
        run(fft, c.kind, after.data(), c.N, c.stride, c.dir);
      }
      // the record's DIR is the sign of the exponent the call applies
      const int sign = c.kind == 1 ? -1 : c.kind == 2 ? 1 : (c.dir == 1 ? 1 : -1);
      record(f, kase * 10 + c.kind, c.N, c.stride, sign, before, after);
      kase++;
    }
  }
  fclose(f);
  printf("fft1d cases: %lld\n", kase);
  upcxx::finalize();
  return 0;
}
