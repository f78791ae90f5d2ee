// Autotuner of the limb-transform launch shapes.  The transform's cost
// depends on the R x C split of N, on the tile each CTA of the column and row
// passes takes, on how many CTAs share a tile column (waves) and on how many
// limbs one launch pair covers (the L2 budget of the column -> row handoff).
// The tuner times forward + inverse transforms of the engine's ring on a
// device buffer far larger than L2 and on batch-sized calls issued from two
// streams at once, and walks the knobs one at a time (coordinate descent),
// keeping a change only when it is at least 2% faster (best of two timings
// per trial).  No reference counterpart: the reference fixes its transform
// shapes at compile time
// (aoa-ntt src/cuda/htrans/ntt.cu:35-65).
#include <cstdio>
#include <cstring>
#include <functional>

#include "aoa_internal.h"

namespace aoa {
namespace {

// residues x < q of limb l, from a counter-based hash (no host transfer)
__global__ void fill_residues(uint64_t* d, long n_per_limb, int nlimbs_per_poly, long total, const PrimeConst* pc) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    uint64_t z = (uint64_t)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const int limb = (int)((i / n_per_limb) % nlimbs_per_poly);
    d[i] = z % pc[limb].q;
  }
}

struct Knob {
  const char* name;
  std::vector<double> values;
  std::function<double(const Tune&)> get;
  std::function<void(Tune&, double)> set;
};

}  // namespace
}  // namespace aoa

using namespace aoa;

extern "C" int aoa_engine_autotune(aoa_engine* h, int limbs, char* report, size_t report_len) {
  if (!h || limbs < 0) return fail(AOA_ERR_BAD_PARAM, "bad argument");
  Engine& E = h->e;
  const Tune saved = E.tune;
  cudaStream_t st = nullptr, st2 = nullptr;
  uint64_t* buf = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr, ef = nullptr, ej = nullptr;
  std::string rep;
  const int st_ = guarded([&] {
    if (E.log_n < 10) throw AoaError(AOA_ERR_BAD_PARAM, "autotune: ring too small for the two-pass transform");
    const long N = E.N;
    const int k = E.k;
    // about 12x the L2 size by default, in whole polys of k limbs
    const long want = limbs > 0 ? limbs : std::max<long>(k, (1536L << 20) / (8 * N));
    const int npolys = (int)std::max<long>(1, (want + k - 1) / k);
    const long words = (long)npolys * k * N;
    AOA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    AOA_CUDA(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
    AOA_CUDA(cudaMalloc(&buf, words * 8));
    AOA_CUDA(cudaEventCreate(&e0));
    AOA_CUDA(cudaEventCreate(&e1));
    AOA_CUDA(cudaEventCreateWithFlags(&ef, cudaEventDisableTiming));
    AOA_CUDA(cudaEventCreateWithFlags(&ej, cudaEventDisableTiming));
    fill_residues<<<4 * E.num_sms, 256, 0, st>>>(buf, N, k, words, E.d_pc);
    AOA_CHECK_LAUNCH();
    // Objective: forward + inverse time per limb on the whole sample plus the
    // same on batch-sized calls (8 polys on each of two streams at once, as
    // the two halves of a batched HMult of 16 run their transforms), so
    // that a shape that only pays off on very large calls does not win.
    // Each figure is the best of two timings.
    const int half = std::max(1, std::min(npolys / 2, 8));
    auto time_polys = [&](int np, int reps, bool two) -> float {
      float best_ms = 0;
      for (int t = 0; t < 3; t++) {                  // warm-up, then two timed runs
        AOA_CUDA(cudaEventRecord(e0, st));
        if (two) {
          AOA_CUDA(cudaEventRecord(ef, st));
          AOA_CUDA(cudaStreamWaitEvent(st2, ef, 0));
        }
        for (int r = 0; r < reps; r++) {
          ntt_batch(E, buf, np, 0, k, k, true, st);
          ntt_batch(E, buf, np, 0, k, k, false, st);
          if (two) {
            uint64_t* b2 = buf + (long)np * k * N;
            ntt_batch(E, b2, np, 0, k, k, true, st2);
            ntt_batch(E, b2, np, 0, k, k, false, st2);
          }
        }
        if (two) {
          AOA_CUDA(cudaEventRecord(ej, st2));
          AOA_CUDA(cudaStreamWaitEvent(st, ej, 0));
        }
        AOA_CUDA(cudaEventRecord(e1, st));
        AOA_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        AOA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (t == 1 || (t == 2 && ms < best_ms)) best_ms = ms;
      }
      return best_ms / reps;
    };
    auto time_once = [&]() -> float {
      return time_polys(npolys, 2, false) + time_polys(half, 4, true) * (float)npolys / (float)(2 * half);
    };
    std::vector<Knob> knobs = {
        {"ntt_split", {0, -1, 1, -2, 2}, [](const Tune& t) { return (double)t.ntt_split; },
         [](Tune& t, double v) { t.ntt_split = (int)v; }},
        {"ntt_cols_div", {0, 1, 2}, [](const Tune& t) { return (double)t.ntt_cols_div; },
         [](Tune& t, double v) { t.ntt_cols_div = (int)v; }},
        {"ntt_cols_kind", {0, 1}, [](const Tune& t) { return (double)t.ntt_cols_kind; },
         [](Tune& t, double v) { t.ntt_cols_kind = (int)v; }},
        {"ntt_rows_div", {0, 1, 2}, [](const Tune& t) { return (double)t.ntt_rows_div; },
         [](Tune& t, double v) { t.ntt_rows_div = (int)v; }},
        {"ntt_waves", {1, 2, 0.5, 4, 8}, [](const Tune& t) { return t.ntt_waves; },
         [](Tune& t, double v) { t.ntt_waves = v; }},
        {"ntt_waves_large", {1, 2, 4, 8, 16}, [](const Tune& t) { return t.ntt_waves_large; },
         [](Tune& t, double v) { t.ntt_waves_large = v; }},
        {"ntt_chunk_bytes", {1024.0 * (1 << 20), 120.0 * (1 << 20), 384.0 * (1 << 20), 4096.0 * (1 << 20)},
         [](const Tune& t) { return (double)t.ntt_chunk_bytes; },
         [](Tune& t, double v) { t.ntt_chunk_bytes = (long)v; }},
    };
    float best = time_once();
    char line[256];
    snprintf(line, sizeof line, "{\"limbs\": %ld, \"start_ms\": %.4f, \"trials\": [", (long)npolys * k, best);
    rep = line;
    bool first = true;
    auto descend = [&](const Knob& kn) {
      const double cur = kn.get(E.tune);
      double keep = cur;
      for (double v : kn.values) {
        if (v == cur) continue;
        kn.set(E.tune, v);
        const float ms = time_once();
        snprintf(line, sizeof line, "%s{\"%s\": %g, \"ms\": %.4f}", first ? "" : ", ", kn.name, v, ms);
        rep += line;
        first = false;
        if (ms < best * 0.98f) {
          best = ms;
          keep = v;
        }
      }
      kn.set(E.tune, keep);
    };
    // two rounds of coordinate descent: a knob's best value can move once the
    // others have changed
    for (int round = 0; round < 2; round++)
      for (const Knob& kn : knobs) descend(kn);
    snprintf(line, sizeof line,
             "], \"best_ms\": %.4f, \"choice\": {\"ntt_split\": %d, \"ntt_cols_div\": %d, \"ntt_cols_kind\": %d, "
             "\"ntt_rows_div\": %d, \"ntt_waves\": %g, \"ntt_waves_large\": %g, \"ntt_chunk_bytes\": %ld}}",
             best, E.tune.ntt_split, E.tune.ntt_cols_div, E.tune.ntt_cols_kind, E.tune.ntt_rows_div, E.tune.ntt_waves,
             E.tune.ntt_waves_large, E.tune.ntt_chunk_bytes);
    rep += line;
  });
  if (st_ != AOA_OK) E.tune = saved;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (ef) cudaEventDestroy(ef);
  if (ej) cudaEventDestroy(ej);
  if (buf) cudaFree(buf);
  if (st) cudaStreamDestroy(st);
  if (st2) cudaStreamDestroy(st2);
  if (report && report_len) {
    const size_t n = std::min(report_len - 1, rep.size());
    memcpy(report, rep.data(), n);
    report[n] = 0;
  }
  return st_;
}
