// TEST INFRASTRUCTURE, not product code. Runs the device LDL^T panel
// (fieldcraft_b200/csrc/cuda/ldlt_panel.cuh) on the CPU, host threads standing for the threads
// of a block and a barrier for __syncthreads, so that tests can check the kernel's source
// against the oracle bit for bit without a GPU. Built with -ffp-contract=off, as the oracle.
//
// The barrier checks that every thread arrives from the same call site the same number of
// times (a thread that took another branch would hang a GPU block); on a mismatch the run stops
// waiting and reports it. Optional jitter delays threads at random after each barrier, so that
// a thread writing what another has yet to read shows up as a wrong bit.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "cuda/ldlt_panel.cuh"

namespace {

class Barrier {
 public:
  explicit Barrier(int count) : count_(count) {}
  void wait() {
    std::unique_lock<std::mutex> lock(mu_);
    const int64_t generation = generation_;
    if (++waiting_ == count_) {
      waiting_ = 0;
      ++generation_;
      cv_.notify_all();
    } else {
      cv_.wait(lock, [&] { return generation_ != generation; });
    }
  }

 private:
  std::mutex mu_;
  std::condition_variable cv_;
  int count_, waiting_ = 0;
  int64_t generation_ = 0;
};

constexpr int MAX_EMULATED = fc::ldlt::MAX_THREADS;

struct Checks {
  const void *site[MAX_EMULATED];
  int64_t count[MAX_EMULATED];
  std::atomic<bool> diverged{false};
  int jitter = 0;  // 0: none; else the seed of the delays
};

struct HostBlock {
  int t, n;
  Barrier *barrier;
  Checks *checks;
  std::mt19937 rng;
  int tid() const { return t; }
  int size() const { return n; }
  __attribute__((noinline)) void sync() {
    if (checks->diverged) return;
    checks->site[t] = __builtin_return_address(0);
    checks->count[t] += 1;
    barrier->wait();
    for (int u = 0; u < n; ++u)
      if (checks->site[u] != checks->site[t] || checks->count[u] != checks->count[t]) checks->diverged = true;
    barrier->wait();
    if (checks->jitter && rng() % 4 == 0) std::this_thread::sleep_for(std::chrono::microseconds(rng() % 40));
  }
};

}  // namespace

extern "C" {

// Factors one front (m x w column-major in F, rows >= columns meaningful) with the panel source
// on `threads` host threads, panel after panel; between panels the later own columns take the
// panel's update over the kernel's update tiles (update_tile), each entry in the oracle's order
// (its sum over the panel's columns from zero, then one subtraction). scale[w]: the largest |A| of each own column. Fills order[w] and pivots[w];
// *twos receives the 2 x 2 pivots. jitter: 0, or a seed for random delays after barriers.
// Returns -1, the own column found singular, -2 when the threads returned different results,
// -3 when they reached different barriers.
int emu_ldlt_front(int64_t m, int w, double *F, const double *scale, int32_t *order, int8_t *pivots, int threads,
                   int jitter, int *twos) {
  namespace L = fc::ldlt;
  if (threads < 1 || threads > MAX_EMULATED) return -2;
  Checks checks;
  checks.jitter = jitter;
  for (int t = 0; t < threads; ++t) checks.count[t] = 0;
  std::vector<double> a(m), b(m), W((size_t)(w > 0 ? w : 1) * (L::PANEL + 1));
  for (int c = 0; c < w; ++c) {
    order[c] = c;
    pivots[c] = L::PIVOT_ONE;
  }
  L::Front f{F, m, w, scale, order, pivots, a.data(), b.data(), W.data(), (int64_t)(w > 0 ? w : 1)};
  L::Shared sh;
  Barrier barrier(threads);
  *twos = 0;
  int c0 = 0;
  while (c0 < w) {
    std::vector<int> result(threads), end(threads), made(threads);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        HostBlock blk{t, threads, &barrier, &checks, std::mt19937((uint32_t)(jitter * 7919 + t + 1000 * c0))};
        int e = c0, x = 0;
        const int r = L::panel(blk, sh, f, c0, &e, &x);
        if (r < 0) L::panel_w(blk, f, c0, e);
        result[t] = r;
        end[t] = e;
        made[t] = x;
      });
    for (auto &th : pool) th.join();
    if (checks.diverged) return -3;
    for (int t = 1; t < threads; ++t)
      if (result[t] != result[0] || (result[0] < 0 && (end[t] != end[0] || made[t] != made[0]))) return -2;
    if (result[0] >= 0) return result[0];
    *twos += made[0];
    // the update tile by tile, as the GEMM tasks the kernel writes would apply it
    const int c1 = end[0], kw = c1 - c0;
    L::Tile tile;
    for (int64_t slot = 0; L::update_tile(m, w, c1, slot, tile); ++slot)
      for (int jj = 0; jj < tile.N; ++jj)
        for (int ii = 0; ii < tile.M; ++ii) {
          const int64_t i = tile.i0 + ii;
          const int c = tile.j0 + jj;
          if (tile.lower && i < c) continue;
          double s = 0.0;
          for (int j = 0; j < kw; ++j) s += F[i + (int64_t)(c0 + j) * m] * W[(c - c1) + (int64_t)j * f.ld_w];
          F[i + (int64_t)c * m] -= s;
        }
    c0 = c1;
  }
  return -1;
}

}  // extern "C"

extern "C" {

// Every update tile of a front (m rows, w own columns) after a panel that ended at c1: rows
// i0[], columns j0[], sizes M[], N[], lower[] for at most cap tiles; returns the count, which
// update_tiles must give.
int64_t emu_update_tiles(int64_t m, int w, int c1, int64_t *i0, int32_t *j0, int32_t *M, int32_t *N, int8_t *lower,
                         int64_t cap) {
  fc::ldlt::Tile t;
  int64_t count = 0;
  for (int64_t slot = 0; fc::ldlt::update_tile(m, w, c1, slot, t); ++slot, ++count)
    if (count < cap) {
      i0[count] = t.i0;
      j0[count] = t.j0;
      M[count] = t.M;
      N[count] = t.N;
      lower[count] = t.lower;
    }
  return count == fc::ldlt::update_tiles(m, w, c1) ? count : -1;
}

}  // extern "C"

extern "C" {

// After a front is factored (emu_ldlt_front): W21 = L21 D into w21 (ld m - w), then D out of the
// front into d and e (split_d), on `threads` host threads. Returns 0, or -3 on a divergence.
int emu_ldlt_after(int64_t m, int w, double *F, const int8_t *pivots, double *w21, double *d, double *e, int threads) {
  namespace L = fc::ldlt;
  if (threads < 1 || threads > MAX_EMULATED) return -2;
  Checks checks;
  for (int t = 0; t < threads; ++t) checks.count[t] = 0;
  L::Front f{F, m, w, nullptr, nullptr, const_cast<int8_t *>(pivots), nullptr, nullptr, nullptr, 0};
  Barrier barrier(threads);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      HostBlock blk{t, threads, &barrier, &checks, std::mt19937((uint32_t)t)};
      L::front_w21(blk, f, w21, m - w > 0 ? m - w : 1);
      L::split_d(blk, f, d, e);
    });
  for (auto &th : pool) th.join();
  return checks.diverged ? -3 : 0;
}

// y <- D^-1 y over n unknowns of R right-hand sides (row-major), one call per pivot group.
void emu_apply_d_inverse(int64_t n, int R, const double *d, const double *e, const int8_t *pivots, double *y) {
  for (int64_t i = 0; i < n; ++i) fc::ldlt::apply_d_inverse(i, R, d, e, pivots, y);
}

}  // extern "C"

extern "C" {

// X = L^-1 of a unit lower nb x nb block (column-major, leading dimensions ldl and ldx) on
// `threads` host threads. Returns 0, or -3 on a divergence.
int emu_unit_lower_inverse(const double *Lb, int64_t ldl, int nb, double *X, int64_t ldx, int threads) {
  if (threads < 1 || threads > MAX_EMULATED) return -2;
  Checks checks;
  for (int t = 0; t < threads; ++t) checks.count[t] = 0;
  Barrier barrier(threads);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      HostBlock blk{t, threads, &barrier, &checks, std::mt19937((uint32_t)t)};
      fc::ldlt::unit_lower_inverse(blk, Lb, ldl, nb, X, ldx);
    });
  for (auto &th : pool) th.join();
  return checks.diverged ? -3 : 0;
}

// The rows below the own columns of an m x w front permuted (row w + i takes old row w + from[i]).
int emu_permute_rows_below(int64_t m, int w, double *F, const int32_t *from, int threads) {
  if (threads < 1 || threads > MAX_EMULATED) return -2;
  Checks checks;
  for (int t = 0; t < threads; ++t) checks.count[t] = 0;
  Barrier barrier(threads);
  std::vector<double> tmp((size_t)(m - w > 0 ? m - w : 1));
  fc::ldlt::Front f{F, m, w, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      HostBlock blk{t, threads, &barrier, &checks, std::mt19937((uint32_t)t)};
      fc::ldlt::permute_rows_below(blk, f, from, tmp.data());
    });
  for (auto &th : pool) th.join();
  return checks.diverged ? -3 : 0;
}

}  // extern "C"
