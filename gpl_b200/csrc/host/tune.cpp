// The in-place autotuner (tune.h).
#include "tune.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>

namespace gpl {

Tuner::Tuner(std::string what, std::vector<std::string> names, const char *env, int probe, int period)
    : what_(std::move(what)), names_(std::move(names)), probe_(std::max(1, probe)), base_period_(std::max(1, period)), period_(std::max(1, period)) {
  n_ = (int)names_.size();
  samples_.assign(n_, {});
  median_.assign(n_, -1.0f);
  if (env)
    if (const char *v = std::getenv(env))
      for (int k = 0; k < n_; k++)
        if (names_[k] == v) fixed_ = k;
  if (fixed_ >= 0) best_ = fixed_;
  probing_ = fixed_ < 0 && n_ > 1;
  if (probing_)
    for (auto &e : ev_)
      if (cudaEventCreate(&e) != cudaSuccess) {
        // no events: the first candidate, untimed (the error is not left for the next call)
        cudaGetLastError();
        probing_ = false;
      }
}

Tuner::~Tuner() {
  for (auto &e : ev_)
    if (e) cudaEventDestroy(e);
}

int Tuner::start(cudaStream_t s) {
  in_flight_ = true;  // a use that was never finished is dropped
  timed_ = false;
  if (fixed_ >= 0) {
    cur_ = fixed_;
  } else if (probing_ && probe_pos_ < n_ * probe_) {
    cur_ = probe_pos_ % n_;  // the candidates interleaved, so a drift in the state hits each alike
    probe_pos_++;
    timed_ = cudaEventRecord(ev_[0], s) == cudaSuccess;
  } else {
    cur_ = best_;
  }
  return cur_;
}

void Tuner::stop(cudaStream_t s) {
  if (timed_ && cudaEventRecord(ev_[1], s) != cudaSuccess) timed_ = false;
}

void Tuner::finish(bool count) {
  if (!in_flight_) return;
  in_flight_ = false;
  if (timed_ && count) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ev_[0], ev_[1]) == cudaSuccess)
      samples_[cur_].push_back(ms);
    else
      cudaGetLastError();
  }
  timed_ = false;
  if (fixed_ >= 0 || n_ < 2) return;
  if (probing_) {
    if (probe_pos_ >= n_ * probe_) decide();
  } else if (++since_ >= period_) {
    probing_ = true;
    probe_pos_ = 0;
    for (auto &v : samples_) v.clear();
  }
}

void Tuner::decide() {
  int pick = -1;
  for (int k = 0; k < n_; k++) {
    auto &v = samples_[k];
    if (v.empty()) continue;
    std::sort(v.begin(), v.end());
    median_[k] = v[v.size() / 2];
    if (pick < 0 || median_[k] < median_[pick]) pick = k;
  }
  if (pick >= 0) {
    period_ = pick == best_ && probes_ > 0 ? std::min(2 * period_, 16 * base_period_) : base_period_;
    best_ = pick;
  }
  probing_ = false;
  since_ = 0;
  probes_++;
}

std::string Tuner::report() const {
  std::string s = what_ + ": " + names_[best_] + (fixed_ >= 0 ? " (fixed)" : "") + " (";
  char buf[32];
  for (int k = 0; k < n_; k++) {
    if (median_[k] < 0)
      std::snprintf(buf, sizeof buf, "%s-", k ? " / " : "");
    else
      std::snprintf(buf, sizeof buf, "%s%.1f", k ? " / " : "", 1000.0 * median_[k]);
    s += buf;
  }
  return s + " us)";
}

}  // namespace gpl
