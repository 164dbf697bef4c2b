// TEST INFRASTRUCTURE ONLY -- stand-in for the absent cdf_timer submodule
// (.gitmodules:5-8 of the reference project): named tic/toc accumulators.
#pragma once
#include <chrono>
#include <cstdio>
#include <map>
#include <string>

namespace cdf {
namespace timer {
class timer_t {
 public:
  void tic(const std::string& k) { start_[k] = std::chrono::steady_clock::now(); }
  void toc(const std::string& k) {
    total_[k] += std::chrono::duration<double>(std::chrono::steady_clock::now() - start_[k]).count();
  }
  void print_report() const {
    for (auto const& kv : total_) std::fprintf(stderr, "timer %-16s %12.6f s\n", kv.first.c_str(), kv.second);
  }

 private:
  std::map<std::string, std::chrono::steady_clock::time_point> start_;
  std::map<std::string, double> total_;
};
}  // namespace timer
}  // namespace cdf
