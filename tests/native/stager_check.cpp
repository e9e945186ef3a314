// Checks of evora::Stager (the serving loop's threaded host copies): copies
// posted back to back complete with the right bytes, copy() helps until its
// own copy is done while others are queued, zero-byte and sub-chunk copies
// complete, and stop() finishes everything queued.  Prints "ok" on success.
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <random>
#include <vector>

#include "../../evora_b200/csrc/stager.h"

static bool check(bool ok, const char* what) {
  if (!ok) std::printf("FAIL: %s\n", what);
  return ok;
}

int main() {
  std::mt19937_64 rng(5);
  const int R = 120;
  std::vector<std::vector<unsigned char>> src(R), dst(R);
  std::vector<std::unique_ptr<std::atomic<int>>> left(R);
  for (int i = 0; i < R; ++i) {
    size_t n = i % 10 == 0 ? 0 : (size_t)(rng() % (11u << 20)) + 1;   // 0 .. 11 MB
    src[i].resize(n);
    for (size_t k = 0; k < n; ++k) src[i][k] = (unsigned char)(rng() >> 56);
    dst[i].assign(n, 0);
    left[i].reset(new std::atomic<int>(0));
  }
  bool ok = true;
  {
    evora::Stager st;
    for (int i = 0; i < R; ++i) {
      st.post(dst[i].data(), src[i].data(), src[i].size(), left[i].get());
      if (i % 17 == 0) {   // a synchronous copy in between, behind the queued ones
        std::vector<unsigned char> a(9u << 20), b(9u << 20, 0);
        for (size_t k = 0; k < a.size(); k += 4096) a[k] = (unsigned char)(k >> 12);
        st.copy(b.data(), a.data(), a.size());
        ok &= check(a == b, "copy() behind queued posts");
      }
    }
    for (int i = 0; i < R; ++i) {
      while (left[i]->load(std::memory_order_acquire) > 0) std::this_thread::yield();
      ok &= check(dst[i] == src[i], "posted copy");
    }
    // stop() with work still queued finishes it
    std::vector<unsigned char> a(13u << 20, 7), b(13u << 20, 0);
    std::atomic<int> l{0};
    st.post(b.data(), a.data(), a.size(), &l);
    st.stop();
    ok &= check(l.load() == 0 && a == b, "stop() drains the queue");
    // small copies go straight through
    unsigned char x[100], y[100] = {0};
    for (int k = 0; k < 100; ++k) x[k] = (unsigned char)k;
    st.copy(y, x, sizeof x);
    ok &= check(std::memcmp(x, y, sizeof x) == 0, "small copy");
  }
  if (ok) std::printf("ok\n");
  return ok ? 0 : 1;
}
