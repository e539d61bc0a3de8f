// A caller without Python: builds a solver from an export folder (include/maxichem_b200.hpp) and makes one call on
// inputs read from raw files, writing the outputs next to them. Test infrastructure for tests/test_gpu_export.py.
//   call_export <export folder> <io folder> <cells>
// io folder: x.bin [B][ns], T.bin, P.bin, dt.bin, h.bin [B], J.bin [B][nj] (float64); writes x_out.bin, h_out.bin,
// steps.bin (float64), done.bin, flag.bin, status.bin, count.bin (int32). Exit 0 on success, 3 when the call refused
// cells (the message on stdout), 2 on other errors.
#include <cuda_runtime.h>

#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "maxichem_b200.hpp"

template <typename T>
std::vector<T> load(const std::string& path, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  if (!f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T)))) throw std::runtime_error(path);
  return v;
}

template <typename T>
void save(const std::string& path, const std::vector<T>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

template <typename T>
T* device(const std::vector<T>& v) {
  T* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(v.size(), 1) * sizeof(T)) != cudaSuccess) throw std::runtime_error("cudaMalloc");
  if (!v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return p;
}

template <typename T>
std::vector<T> host(const T* p, size_t n) {
  std::vector<T> v(n);
  cudaMemcpy(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost);
  return v;
}

int main(int argc, char** argv) {
  if (argc != 4) {
    std::cerr << "usage: call_export <export folder> <io folder> <cells>\n";
    return 2;
  }
  const std::string io = argv[2];
  const size_t B = std::stoul(argv[3]);
  try {
    maxichem_b200::Solver chem(argv[1], 0);
    const size_t ns = (size_t)chem.ns(), nj = (size_t)chem.nj();
    double* x = device(load<double>(io + "/x.bin", B * ns));
    double* T = device(load<double>(io + "/T.bin", B));
    double* P = device(load<double>(io + "/P.bin", B));
    double* dt = device(load<double>(io + "/dt.bin", B));
    double* h = device(load<double>(io + "/h.bin", B));
    double* J = nj ? device(load<double>(io + "/J.bin", B * nj)) : nullptr;
    double* xo = device(std::vector<double>(B * ns));
    double* ho = device(std::vector<double>(B));
    double* steps = device(std::vector<double>(B));
    int32_t* done = device(std::vector<int32_t>(B));
    int32_t* flag = device(std::vector<int32_t>(B));
    int32_t* status = device(std::vector<int32_t>(B));
    int rc = 0;
    try {
      chem(x, T, P, dt, h, J, (int64_t)B, xo, ho, done, steps, flag, status);
      std::cout << "ok " << chem.species().size() << " species\n";
    } catch (std::invalid_argument const& e) {
      std::cout << "refused: " << e.what() << "\n";
      rc = 3;
    }
    save(io + "/x_out.bin", host(xo, B * ns));
    save(io + "/h_out.bin", host(ho, B));
    save(io + "/steps.bin", host(steps, B));
    save(io + "/done.bin", host(done, B));
    save(io + "/flag.bin", host(flag, B));
    save(io + "/status.bin", host(status, B));
    save(io + "/count.bin", chem.count());
    for (void* p : {(void*)x, (void*)T, (void*)P, (void*)dt, (void*)h, (void*)J, (void*)xo, (void*)ho, (void*)steps,
                    (void*)done, (void*)flag, (void*)status})
      if (p) cudaFree(p);
    return rc;
  } catch (std::exception const& e) {
    std::cout << "error: " << e.what() << "\n";
    return 2;
  }
}
