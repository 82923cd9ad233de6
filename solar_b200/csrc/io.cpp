// io.cpp -- the reference's output files, written (and the restart also read) in its byte
// and text layouts, for one zone at a time from host arrays.  The context-level entry
// points in solar_gpu.cu gather the needed data from the device and call these.
//
//   restart   output.f90:86-190   MPI-IO file 'Restart/restart.NNN.<zone>': header of four
//                                 default integers (nx, ny, nr, 5), time (real*8) and step
//                                 (integer), then q(nx,ny,nr,5) real*8 in Fortran order at
//                                 byte 28 (disp = 5*intSize + realSize).  The reference has
//                                 only the writer; the reader here accepts the same layout.
//   visual    output.f90:192-240  Fortran unformatted sequential record of q(:,:,o_rad,1:5)
//                                 in 'Visual/NNN/vis_<rank>' (record markers: 4-byte lengths).
//   grid      output.f90:242-267  'Visual/grid/grid_<rank>', FORMAT(1x, 7i5).
//   forcing   output.f90:271-307  'forcing/forcing_cubesph.<zone>' (read only): one record of
//                                 f(nx, ny, nt) with n fastest.
//   trace     output.f90:309-343  'trace_<zone>', appended, ((q(1,1,k,l), k=1,mr), l=1,5)
//                                 with FORMAT(1x, 5(ES13.5)): five values per line, the
//                                 leading blank on the first line only (format reversion).
#include <sys/stat.h>
#include <sys/types.h>

#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/solar_gpu.h"

namespace solar {
int report_error(int code, const char* msg);
}

namespace {

int io_fail(const std::string& m) { return solar::report_error(SOLAR_ERR_ARG, m.c_str()); }

// mkdir -p for the directories of `path` (the last component is a file name)
int make_parents(const std::string& path) {
  for (size_t p = path.find('/', 1); p != std::string::npos; p = path.find('/', p + 1)) {
    const std::string d = path.substr(0, p);
    if (mkdir(d.c_str(), 0775) != 0 && errno != EEXIST) return io_fail("cannot create directory " + d);
  }
  return SOLAR_OK;
}

}  // namespace

extern "C" {

// The three-digit cue of the reference's directory and file names (dirs.c:20, output.f90:121-127).
int solar_io_cue_name(int cue, char* buf, int len) {
  if (!buf || len <= 0 || cue < 0) return io_fail("bad cue or buffer");
  std::snprintf(buf, (size_t)len, "%d%d%d", cue / 100, (cue % 100) / 10, cue % 10);
  return SOLAR_OK;
}

// Fortran ESw.d edit descriptor: optional sign, one digit, '.', d digits, then E+zz for
// |exponent| <= 99 or +zzz for |exponent| <= 999, right-justified in w characters; a value
// that does not fit prints w asterisks.
int solar_io_format_es(double v, int w, int d, char* out) {
  if (!out || w <= 0 || d < 0 || w > 60 || d > 40) return io_fail("bad ES descriptor");
  char field[160];
  if (std::isnan(v)) std::snprintf(field, sizeof field, "NaN");
  else if (std::isinf(v)) std::snprintf(field, sizeof field, "%sInfinity", v < 0 ? "-" : "");
  else {
    char buf[96];
    std::snprintf(buf, sizeof buf, "%.*E", d, v);
    char* e = std::strchr(buf, 'E');
    const int ex = std::atoi(e + 1);
    *e = '\0';
    const int ax = ex < 0 ? -ex : ex;
    if (ax <= 99) std::snprintf(field, sizeof field, "%sE%c%02d", buf, ex < 0 ? '-' : '+', ax);
    else std::snprintf(field, sizeof field, "%s%c%03d", buf, ex < 0 ? '-' : '+', ax);
  }
  const int len = (int)std::strlen(field);
  if (len > w) {
    std::memset(out, '*', (size_t)w);
  } else {
    std::memset(out, ' ', (size_t)(w - len));
    std::memcpy(out + (w - len), field, (size_t)len);
  }
  out[w] = '\0';
  return SOLAR_OK;
}

int solar_io_write_restart(const char* path, const double* q, int nx, int ny, int nr, double time, int step) {
  if (!path || !q || nx < 1 || ny < 1 || nr < 1) return io_fail("bad restart arguments");
  if (make_parents(path)) return SOLAR_ERR_ARG;
  FILE* f = std::fopen(path, "wb");
  if (!f) return io_fail(std::string("cannot open ") + path);
  const int32_t gs[4] = {nx, ny, nr, 5};
  const int32_t st = step;
  const size_t n = (size_t)nx * ny * nr * 5;
  bool ok = std::fwrite(gs, sizeof gs, 1, f) == 1 && std::fwrite(&time, sizeof time, 1, f) == 1 &&
            std::fwrite(&st, sizeof st, 1, f) == 1 && std::fwrite(q, sizeof(double), n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? SOLAR_OK : io_fail(std::string("write failed: ") + path);
}

int solar_io_read_restart(const char* path, double* q, int nx, int ny, int nr, double* time, int* step) {
  if (!path || !q) return io_fail("bad restart arguments");
  FILE* f = std::fopen(path, "rb");
  if (!f) return io_fail(std::string("cannot open ") + path);
  int32_t gs[4];
  double t = 0;
  int32_t st = 0;
  const size_t n = (size_t)nx * ny * nr * 5;
  bool ok = std::fread(gs, sizeof gs, 1, f) == 1 && std::fread(&t, sizeof t, 1, f) == 1 &&
            std::fread(&st, sizeof st, 1, f) == 1;
  if (ok && (gs[0] != nx || gs[1] != ny || gs[2] != nr || gs[3] != 5)) {
    std::fclose(f);
    char m[256];
    std::snprintf(m, sizeof m, "%s holds a %d x %d x %d x %d state, expected %d x %d x %d x 5", path, gs[0], gs[1],
                  gs[2], gs[3], nx, ny, nr);
    return io_fail(m);
  }
  ok = ok && std::fread(q, sizeof(double), n, f) == n;
  std::fclose(f);
  if (!ok) return io_fail(std::string("short restart file ") + path);
  if (time) *time = t;
  if (step) *step = st;
  return SOLAR_OK;
}

// READ_FORCING_FUNC (output.f90:271-307): 'forcing/forcing_cubesph.<zone>', one unformatted
// sequential record of f(nx, ny, nt) written with n fastest, then j, then i.  `f` receives
// the record as stored: f[(i*ny + j)*nt + n].
int solar_io_read_forcing(const char* path, int nx, int ny, int nt, double* f) {
  if (!path || !f || nx < 1 || ny < 1 || nt < 1) return io_fail("bad forcing arguments");
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return io_fail(std::string("cannot open ") + path);
  const size_t n = (size_t)nx * ny * nt;
  int32_t head = 0, tail = 0;
  bool ok = std::fread(&head, sizeof head, 1, fp) == 1 && (size_t)head == n * sizeof(double) &&
            std::fread(f, sizeof(double), n, fp) == n && std::fread(&tail, sizeof tail, 1, fp) == 1 && tail == head;
  std::fclose(fp);
  if (!ok) {
    char m[256];
    std::snprintf(m, sizeof m, "%s is not one record of %d x %d x %d float64 values", path, nx, ny, nt);
    return io_fail(m);
  }
  return SOLAR_OK;
}

int solar_io_write_visual(const char* path, const double* plane5, int nx, int ny) {
  if (!path || !plane5 || nx < 1 || ny < 1) return io_fail("bad visual arguments");
  if (make_parents(path)) return SOLAR_ERR_ARG;
  FILE* f = std::fopen(path, "wb");
  if (!f) return io_fail(std::string("cannot open ") + path);
  const size_t n = (size_t)nx * ny * 5;
  const int32_t marker = (int32_t)(n * sizeof(double));
  bool ok = std::fwrite(&marker, sizeof marker, 1, f) == 1 && std::fwrite(plane5, sizeof(double), n, f) == n &&
            std::fwrite(&marker, sizeof marker, 1, f) == 1;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? SOLAR_OK : io_fail(std::string("write failed: ") + path);
}

int solar_io_write_grid(const char* path, const int* seven) {
  if (!path || !seven) return io_fail("bad grid arguments");
  if (make_parents(path)) return SOLAR_ERR_ARG;
  FILE* f = std::fopen(path, "w");
  if (!f) return io_fail(std::string("cannot open ") + path);
  std::fprintf(f, " %5d%5d%5d%5d%5d%5d%5d\n", seven[0], seven[1], seven[2], seven[3], seven[4], seven[5], seven[6]);
  return std::fclose(f) == 0 ? SOLAR_OK : io_fail(std::string("write failed: ") + path);
}

int solar_io_append_trace(const char* path, const double* values, int count) {
  if (!path || !values || count < 0) return io_fail("bad trace arguments");
  if (make_parents(path)) return SOLAR_ERR_ARG;
  FILE* f = std::fopen(path, "a");
  if (!f) return io_fail(std::string("cannot open ") + path);
  // Format reversion (Fortran 2008 10.4) returns to the group 5(ES13.5) for every record
  // after the first, so only the first line carries the 1x blank.
  char cell[64];
  for (int q = 0; q < count; ++q) {
    if (q == 0) std::fputc(' ', f);
    solar_io_format_es(values[q], 13, 5, cell);
    std::fputs(cell, f);
    if (q % 5 == 4 || q == count - 1) std::fputc('\n', f);
  }
  return std::fclose(f) == 0 ? SOLAR_OK : io_fail(std::string("write failed: ") + path);
}

}  // extern "C"
