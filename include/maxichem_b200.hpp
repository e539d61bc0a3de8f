// maxichem_b200 from C++ with no Python: a solver built from a folder that CudaSolver.export wrote, called on device
// arrays. The counterpart of the reference's maxichem::Solver (cpp/maxichem.hpp:48-94), over plain CUDA device
// pointers instead of libtorch tensors:
//
//   maxichem_b200::Solver chem("export/chno69", 0);
//   chem(x, T, P, dt, h, J, B, x_out, h_out, done, steps, flag, status, stream);
//
// x [B][ns] mole fractions in the network's species order (species()), T [B] K, P [B] dyn cm^-2, dt [B] s, h [B]
// the starting step sizes, J [B][nj] s^-1 (nullptr when nj() == 0); outputs x_out [B][ns], h_out [B], done [B]
// (int32 0/1), steps [B] (float64), flag [B] (int32 0/1/2), status [B] (int32). All are float64 unless stated, on the
// solver's device. A call runs on `stream`, reads its counts back (its one host synchronisation) and throws
// std::invalid_argument if it refused a cell (bad input, or T outside [t_min, t_max]), naming the counts and the first
// such cell; the counts stay readable. The constructor throws std::runtime_error if the export cannot be read.
// Calls share the solver's scratch and counts, so they run one at a time, as in Python.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "maxichem_b200.h"

namespace maxichem_b200 {

inline constexpr double kDefaultRtol = 1e-3;  // DEFAULT_RTOL of maxichem_b200/constants.py
inline constexpr int kDefaultMaxSteps = 4000;  // DEFAULT_MAX_STEPS

class Solver {
 public:
  Solver(std::string const& folder, int device) : device_(device) {
    std::ifstream meta(folder + "/meta.txt");
    if (!meta) throw std::runtime_error("maxichem_b200: " + folder + "/meta.txt cannot be read");
    std::string line;
    while (std::getline(meta, line)) {
      std::istringstream in(line);
      std::string key;
      in >> key;
      if (key == "ns") in >> ns_;
      if (key == "nj") in >> nj_;
      if (key == "atol") in >> default_atol_;
      if (key == "t_min") in >> t_min_;
      if (key == "t_max") in >> t_max_;
      if (key == "x_sum_tol") in >> x_sum_tol_;
      if (key == "species" || key == "elements") {
        std::vector<std::string>& names = key == "species" ? species_ : elements_;
        for (std::string w; in >> w;) names.push_back(w);
      }
    }
    char err[1024] = {0};
    if (mx_create_from_export(folder.c_str(), device, &s_, err, sizeof err) != MX_OK)
      throw std::runtime_error(err);
    int old = 0;
    cudaGetDevice(&old);
    cudaSetDevice(device_);
    const bool ok = cudaMalloc(&count_, MX_COUNT_SLOTS * sizeof(int32_t)) == cudaSuccess &&
                    cudaMalloc(&total_, MX_COUNT_SLOTS * sizeof(int64_t)) == cudaSuccess &&
                    cudaMemset(total_, 0, MX_COUNT_SLOTS * sizeof(int64_t)) == cudaSuccess;
    cudaSetDevice(old);
    if (!ok) {
      release();
      throw std::runtime_error("maxichem_b200: the count arrays cannot be allocated");
    }
  }
  ~Solver() { release(); }
  Solver(Solver const&) = delete;
  Solver& operator=(Solver const&) = delete;

  void operator()(const double* x, const double* T, const double* P, const double* dt, const double* h,
                  const double* J, int64_t B, double* x_out, double* h_out, int32_t* done, double* steps,
                  int32_t* flag, int32_t* status, cudaStream_t stream = nullptr, double rtol = kDefaultRtol,
                  double atol = -1.0, int max_steps = kDefaultMaxSteps) {
    char err[1024] = {0};
    if (atol < 0.0) atol = default_atol_;
    if (mx_call(s_, x, T, P, dt, h, J, B, rtol, atol, max_steps, x_out, h_out, done, steps, flag, status, count_,
                total_, stream, err, sizeof err) != MX_OK)
      throw std::invalid_argument(err);
    const std::vector<int32_t> n = count(stream);
    if (n[MX_COUNT_BAD_INPUT] || n[MX_COUNT_COLD] || n[MX_COUNT_HOT]) refuse(n, status, B, stream);
  }

  int ns() const { return ns_; }
  int nj() const { return nj_; }
  std::vector<std::string> const& species() const { return species_; }
  std::vector<std::string> const& elements() const { return elements_; }
  double default_atol() const { return default_atol_; }
  // the last call's counts (queue, bad_input, cold, hot, nonfinite, unfinished, drift, recomputed, recovered,
  // still_failed, nonfinite_h, the recovery's queue), copied to the host after `stream`
  std::vector<int32_t> count(cudaStream_t stream = nullptr) const {
    std::vector<int32_t> v(MX_COUNT_SLOTS);
    copy(v.data(), count_, sizeof(int32_t) * v.size(), stream);
    return v;
  }
  // their sum since construction
  std::vector<int64_t> total(cudaStream_t stream = nullptr) const {
    std::vector<int64_t> v(MX_COUNT_SLOTS);
    copy(v.data(), total_, sizeof(int64_t) * v.size(), stream);
    return v;
  }
  mx_solver* handle() const { return s_; }

 private:
  int device_ = 0, ns_ = 0, nj_ = 0;
  double default_atol_ = 1e-25, t_min_ = 300.0, t_max_ = 3000.0, x_sum_tol_ = 1e-10;
  std::vector<std::string> species_, elements_;
  mx_solver* s_ = nullptr;
  int32_t* count_ = nullptr;
  int64_t* total_ = nullptr;

  void release() {
    int old = 0;
    cudaGetDevice(&old);
    cudaSetDevice(device_);
    if (count_) cudaFree(count_);
    if (total_) cudaFree(total_);
    cudaSetDevice(old);
    count_ = nullptr;
    total_ = nullptr;
    mx_destroy(s_);
    s_ = nullptr;
  }

  void copy(void* dst, const void* src, size_t bytes, cudaStream_t stream) const {
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      throw std::runtime_error("maxichem_b200: the counts cannot be read back");
  }

  // the refusal of a call (the Python call's _refuse): the counts, the limits and the first refused cell of each kind
  void refuse(std::vector<int32_t> const& n, int32_t* status, int64_t B, cudaStream_t stream) const {
    std::vector<int32_t> st((size_t)B);
    copy(st.data(), status, sizeof(int32_t) * st.size(), stream);
    auto first = [&](int32_t code) {
      for (int64_t i = 0; i < B; i++)
        if (st[(size_t)i] == code) return i;
      return (int64_t)-1;
    };
    std::ostringstream msg;
    msg << "the call refused cells:";
    if (n[MX_COUNT_COLD])
      msg << " " << n[MX_COUNT_COLD] << " cells below " << t_min_ << " K (first: cell " << first(MX_REFUSED_COLD)
          << ");";
    if (n[MX_COUNT_HOT])
      msg << " " << n[MX_COUNT_HOT] << " cells above " << t_max_ << " K (first: cell " << first(MX_REFUSED_HOT)
          << ");";
    if (n[MX_COUNT_BAD_INPUT])
      msg << " " << n[MX_COUNT_BAD_INPUT] << " cells of bad input: x negative or non-finite, |sum(x) - 1| above "
          << x_sum_tol_ << " or no x above 0; T non-finite, P non-finite, not above 0 or so large that P / (k_B T) "
          << "overflows, dt negative or non-finite, or J negative or non-finite (first: cell "
          << first(MX_REFUSED_BAD_INPUT) << ");";
    throw std::invalid_argument(msg.str());
  }
};

}  // namespace maxichem_b200
