// restart.cpp -- the reference's on-disk formats: the grid file, the solution
// (restart) file and filestat, read and written on the host (no CUDA calls).
// desalm_checkpoint_* in desalm.cu join them to a context's device state.
//
// Grid and solution files are Fortran unformatted sequential files: each
// record is a 4-byte little-endian byte count, the payload, and the same
// count again.  Values are FP32 (the reference's real(rdf), src/precision.F90:11),
// i fastest, one block.  Host arrays here use the ABI's layouts: q as
// (1:5, i, j, k) with the component fastest (desalm_set_state), grids and
// nu_t as (i, j, k).  me = 4 for a laminar case, 5 with Spalart-Allmaras.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "desalm.h"

namespace {

thread_local std::string g_io_err;

int fail(const std::string& msg) {
  g_io_err = msg;
  return DESALM_EIO;
}

struct File {
  FILE* f = nullptr;
  std::string path;
  ~File() {
    if (f) fclose(f);
  }
};

int open_file(File& F, const char* path, const char* mode) {
  if (!path) return fail("null path");
  F.path = path;
  F.f = fopen(path, mode);
  if (!F.f) return fail(std::string("cannot open ") + path + ": " + strerror(errno));
  return 0;
}

// One record of n FP32 values.
int write_record(File& F, const float* v, size_t n) {
  const uint64_t bytes = uint64_t(n) * 4;
  if (bytes > 0x7fffffffull) return fail("record of " + std::to_string(n) + " values exceeds a 4-byte record marker");
  const int32_t m = int32_t(bytes);
  if (fwrite(&m, 4, 1, F.f) != 1 || (n && fwrite(v, 4, n, F.f) != n) || fwrite(&m, 4, 1, F.f) != 1)
    return fail("write to " + F.path + " failed");
  return 0;
}

// Read the next record's length (its leading marker).
int peek_record(File& F, int32_t* bytes) {
  long pos = ftell(F.f);
  if (fread(bytes, 4, 1, F.f) != 1) return fail(F.path + ": unexpected end of file");
  fseek(F.f, pos, SEEK_SET);
  return 0;
}

// Read one record that must hold exactly n FP32 values.
int read_record(File& F, float* v, size_t n, int index) {
  int32_t a = 0, b = 0;
  if (fread(&a, 4, 1, F.f) != 1) return fail(F.path + ": record " + std::to_string(index) + " missing");
  if (int64_t(a) != int64_t(n) * 4)
    return fail(F.path + ": record " + std::to_string(index) + " holds " + std::to_string(a) + " bytes, expected " +
                std::to_string(int64_t(n) * 4));
  if (n && fread(v, 4, n, F.f) != n) return fail(F.path + ": record " + std::to_string(index) + " truncated");
  if (fread(&b, 4, 1, F.f) != 1 || b != a)
    return fail(F.path + ": record " + std::to_string(index) + " has a bad trailing marker");
  return 0;
}

// Close a file that was written, reporting a failed flush.
int finish(File& F) {
  const int r = fclose(F.f);
  F.f = nullptr;
  if (r != 0) return fail("write to " + F.path + " failed");
  return 0;
}

int check_dims(int im, int jm, int km) {
  if (im < 1 || jm < 1 || km < 1) return fail("grid extents must be positive");
  if (int64_t(im) * jm * km * 4 > 0x7fffffffll) return fail("grid too large for 4-byte record markers");
  return 0;
}

}  // namespace

extern "C" {

const char* desalm_io_error(void) { return g_io_err.c_str(); }

int desalm_grid_write(const char* path, int im, int jm, int km, int turbulence, const double* x, const double* y,
                      const double* z, const double* wd) {
  if (int r = check_dims(im, jm, km)) return r;
  if (!x || !y || !z || (turbulence && !wd)) return fail("grid_write: null array");
  const size_t N = size_t(im) * jm * km;
  File F;
  if (int r = open_file(F, path, "wb")) return r;
  std::vector<float> t(N);
  const double* arrs[4] = {x, y, z, wd};
  for (int a = 0; a < (turbulence ? 4 : 3); ++a) {
    for (size_t l = 0; l < N; ++l) t[l] = float(arrs[a][l]);
    if (int r = write_record(F, t.data(), N)) return r;
  }
  return finish(F);
}

int desalm_grid_read(const char* path, int im, int jm, int km, int turbulence, double* x, double* y, double* z,
                     double* wd) {
  if (int r = check_dims(im, jm, km)) return r;
  if (!x || !y || !z || (turbulence && !wd)) return fail("grid_read: null array");
  const size_t N = size_t(im) * jm * km;
  File F;
  if (int r = open_file(F, path, "rb")) return r;
  std::vector<float> t(N);
  double* arrs[4] = {x, y, z, wd};
  for (int a = 0; a < (turbulence ? 4 : 3); ++a) {
    if (int r = read_record(F, t.data(), N, a + 1)) return r;
    for (size_t l = 0; l < N; ++l) arrs[a][l] = double(t[l]);
  }
  return 0;
}

int desalm_solu_write(const char* path, int im, int jm, int km, int turbulence, const double* q, const double* qn,
                      const double* nut) {
  if (int r = check_dims(im, jm, km)) return r;
  if (!q || !qn || (turbulence && !nut)) return fail("solu_write: null array");
  const int me = turbulence ? 5 : 4;
  const size_t N = size_t(im) * jm * km;
  File F;
  if (int r = open_file(F, path, "wb")) return r;
  std::vector<float> t(N);
  // q(1..me), nu_t when turbulent, qn(1..me): one record each
  for (int m = 0; m < me; ++m) {
    for (size_t l = 0; l < N; ++l) t[l] = float(q[5 * l + m]);
    if (int r = write_record(F, t.data(), N)) return r;
  }
  if (turbulence) {
    for (size_t l = 0; l < N; ++l) t[l] = float(nut[l]);
    if (int r = write_record(F, t.data(), N)) return r;
  }
  for (int m = 0; m < me; ++m) {
    for (size_t l = 0; l < N; ++l) t[l] = float(qn[5 * l + m]);
    if (int r = write_record(F, t.data(), N)) return r;
  }
  return finish(F);
}

int desalm_solu_read(const char* path, int im, int jm, int km, int turbulence, double* q, double* qn, double* nut) {
  if (int r = check_dims(im, jm, km)) return r;
  if (!q || !qn) return fail("solu_read: null array");
  const int me = turbulence ? 5 : 4;
  const size_t N = size_t(im) * jm * km;
  File F;
  if (int r = open_file(F, path, "rb")) return r;
  for (size_t l = 0; l < 5 * N; ++l) { q[l] = 0.0; qn[l] = 0.0; }
  std::vector<float> t(size_t(me) * N);
  int32_t first = 0;
  if (int r = peek_record(F, &first)) return r;
  if (!turbulence && int64_t(first) == int64_t(me) * N * 4) {
    // laminar file as the reference reads it: q(1..me) in one record, then qn
    double* dst[2] = {q, qn};
    for (int a = 0; a < 2; ++a) {
      if (int r = read_record(F, t.data(), size_t(me) * N, a + 1)) return r;
      for (int m = 0; m < me; ++m)
        for (size_t l = 0; l < N; ++l) dst[a][5 * l + m] = double(t[size_t(m) * N + l]);
    }
    return 0;
  }
  // one record per component: q(1..me), nu_t when turbulent, qn(1..me)
  int rec = 0;
  for (int m = 0; m < me; ++m) {
    if (int r = read_record(F, t.data(), N, ++rec)) return r;
    for (size_t l = 0; l < N; ++l) q[5 * l + m] = double(t[l]);
  }
  if (turbulence) {
    if (int r = read_record(F, t.data(), N, ++rec)) return r;
    if (nut)
      for (size_t l = 0; l < N; ++l) nut[l] = double(t[l]);
  }
  for (int m = 0; m < me; ++m) {
    if (int r = read_record(F, t.data(), N, ++rec)) return r;
    for (size_t l = 0; l < N; ++l) qn[5 * l + m] = double(t[l]);
  }
  return 0;
}

int desalm_filestat_write(const char* path, double time, int ntime, const double* angle, int n_tur) {
  if (n_tur < 0 || (n_tur > 0 && !angle)) return fail("filestat_write: bad turbine angles");
  File F;
  if (int r = open_file(F, path, "w")) return r;
  // list-directed records: time and step on the first line, one angle a line
  if (fprintf(F.f, " %.9g %d\n", time, ntime) < 0) return fail("write to " + F.path + " failed");
  for (int n = 0; n < n_tur; ++n)
    if (fprintf(F.f, " %.9g\n", angle[n]) < 0) return fail("write to " + F.path + " failed");
  return finish(F);
}

int desalm_filestat_read(const char* path, double* time, int* ntime, double* angle, int n_tur) {
  if (!time || !ntime || n_tur < 0 || (n_tur > 0 && !angle)) return fail("filestat_read: bad arguments");
  File F;
  if (int r = open_file(F, path, "r")) return r;
  if (fscanf(F.f, "%lf %d", time, ntime) != 2) return fail(F.path + ": cannot read time and step");
  const double two_pi = 2.0 * 3.14159265358979323846;
  for (int n = 0; n < n_tur; ++n) {
    if (fscanf(F.f, "%lf", &angle[n]) != 1) return fail(F.path + ": cannot read turbine angle " + std::to_string(n + 1));
    if (angle[n] >= two_pi) angle[n] -= two_pi;  // src/init.F90:272-274
  }
  return 0;
}

}  // extern "C"
