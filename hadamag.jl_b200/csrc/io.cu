// io.cu -- load_state straight into pinned host memory (src/State.jl:388-404).
//
// The reference reads .jld2 (JLD2.load(path, "state")), .npy (NPZ.npzread) or a text file
// of whitespace-separated real / imaginary pairs into a Vector{ComplexF64}.  Here the
// amplitudes land in page-locked memory from cudaMallocHost, so the state's first copy to
// a GPU runs at full link speed and can be asynchronous; .npy files are read with one
// fread into that buffer.  .jld2 (an HDF5 container) is not read: this library links no
// HDF5 implementation.
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "hm_ctx.h"

namespace {

thread_local std::string g_io_err;

int io_fail(int code, const std::string &msg) {
  g_io_err = msg;
  return code;
}

bool is_power(uint64_t len, int q) {
  if (len < 1) return false;
  while (len % (uint64_t)q == 0) len /= (uint64_t)q;
  return len == 1;
}

// value of key 'name' in a .npy header dict, as the raw text up to the next top-level comma
std::string npy_field(const std::string &h, const char *name) {
  const std::string key = std::string("'") + name + "'";
  size_t p = h.find(key);
  if (p == std::string::npos) return "";
  p = h.find(':', p);
  if (p == std::string::npos) return "";
  ++p;
  while (p < h.size() && isspace((unsigned char)h[p])) ++p;
  size_t e = p;
  if (e < h.size() && h[e] == '(') {
    e = h.find(')', e);
    return e == std::string::npos ? "" : h.substr(p, e - p + 1);
  }
  while (e < h.size() && h[e] != ',' && h[e] != '}') ++e;
  return h.substr(p, e - p);
}

int load_npy(FILE *f, double **out, uint64_t *len) {
  unsigned char magic[8];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "\x93NUMPY", 6) != 0)
    return io_fail(HM_ERR_ARG, "not a .npy file (bad magic)");
  uint32_t hlen = 0;
  if (magic[6] == 1) {
    unsigned char b[2];
    if (fread(b, 1, 2, f) != 2) return io_fail(HM_ERR_ARG, "truncated .npy header");
    hlen = b[0] | (b[1] << 8);
  } else {
    unsigned char b[4];
    if (fread(b, 1, 4, f) != 4) return io_fail(HM_ERR_ARG, "truncated .npy header");
    hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
  }
  std::string h(hlen, '\0');
  if (fread(&h[0], 1, hlen, f) != hlen) return io_fail(HM_ERR_ARG, "truncated .npy header");
  const std::string descr = npy_field(h, "descr"), shape = npy_field(h, "shape");
  const bool cplx = descr.find("<c16") != std::string::npos || descr.find("=c16") != std::string::npos;
  const bool real = descr.find("<f8") != std::string::npos || descr.find("=f8") != std::string::npos;
  if (!cplx && !real) return io_fail(HM_ERR_ARG, "only complex128 or float64 .npy vectors are read (descr " + descr + ")");
  // shape: (N,) or (N, 1) / (1, N)
  uint64_t count = 1;
  int dims = 0;
  for (size_t p = 0; p < shape.size();) {
    if (isdigit((unsigned char)shape[p])) {
      char *end = nullptr;
      const unsigned long long v = strtoull(shape.c_str() + p, &end, 10);
      count *= v;
      ++dims;
      p = end - shape.c_str();
    } else {
      ++p;
    }
  }
  if (dims == 0) return io_fail(HM_ERR_ARG, "the .npy array has no elements");
  double *buf = nullptr;
  if (cudaMallocHost((void **)&buf, count * 2 * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return io_fail(HM_ERR_OOM, "cudaMallocHost failed");
  }
  if (cplx) {
    if (fread(buf, sizeof(double), 2 * count, f) != 2 * count) {
      cudaFreeHost(buf);
      return io_fail(HM_ERR_ARG, "truncated .npy data");
    }
  } else {
    // real vector: read into the upper half, then spread to (re, 0) pairs from the front
    double *re = buf + count;
    if (fread(re, sizeof(double), count, f) != count) {
      cudaFreeHost(buf);
      return io_fail(HM_ERR_ARG, "truncated .npy data");
    }
    for (uint64_t i = 0; i < count; ++i) {
      const double v = re[i];
      buf[2 * i] = v;
      buf[2 * i + 1] = 0.0;
    }
  }
  *out = buf;
  *len = count;
  return HM_OK;
}

int load_text(FILE *f, double **out, uint64_t *len) {
  std::vector<double> vals;
  char word[128];
  while (fscanf(f, "%127s", word) == 1) {
    char *end = nullptr;
    const double v = strtod(word, &end);
    if (end == word || *end != '\0') return io_fail(HM_ERR_ARG, std::string("not a number: ") + word);
    vals.push_back(v);
  }
  if (vals.size() % 2 != 0) return io_fail(HM_ERR_ARG, "File does not contain real/imaginary pairs");
  const uint64_t count = vals.size() / 2;
  double *buf = nullptr;
  if (cudaMallocHost((void **)&buf, std::max<size_t>(1, vals.size()) * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return io_fail(HM_ERR_OOM, "cudaMallocHost failed");
  }
  memcpy(buf, vals.data(), vals.size() * sizeof(double));
  *out = buf;
  *len = count;
  return HM_OK;
}

}  // namespace

extern "C" {

int hm_load_state(const char *path, int q, double **psi_pinned, uint64_t *len) {
  g_io_err.clear();
  if (!path || !psi_pinned || !len) return io_fail(HM_ERR_ARG, "null pointer");
  if (q < 2) return io_fail(HM_ERR_ARG, "Base q must be >= 2");
  *psi_pinned = nullptr;
  *len = 0;
  const size_t L = strlen(path);
  if (L >= 5 && strcmp(path + L - 5, ".jld2") == 0)
    return io_fail(HM_ERR_ARG, ".jld2 states are HDF5 files, which this library does not read; save as .npy");
  FILE *f = fopen(path, "rb");
  if (!f) return io_fail(HM_ERR_ARG, std::string("cannot open ") + path);
  double *buf = nullptr;
  uint64_t count = 0;
  const bool npy = L >= 4 && strcmp(path + L - 4, ".npy") == 0;
  const int rc = npy ? load_npy(f, &buf, &count) : load_text(f, &buf, &count);
  fclose(f);
  if (rc != HM_OK) return rc;
  if (!is_power(count, q)) {
    cudaFreeHost(buf);
    return io_fail(HM_ERR_SIZE, "length(vec)=" + std::to_string(count) + " is not a power of q=" + std::to_string(q));
  }
  *psi_pinned = buf;
  *len = count;
  return HM_OK;
}

int hm_free_state(double *psi_pinned) {
  if (psi_pinned) cudaFreeHost(psi_pinned);
  return HM_OK;
}

const char *hm_io_last_error(void) { return g_io_err.c_str(); }

}  // extern "C"
