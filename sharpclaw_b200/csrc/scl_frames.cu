// scl_frames.cu -- frame output compatible with the reference's
// src/1d/out1.f90 and src/2d/out2.f90, so runs stay readable by the Clawpack
// plotting tools.  Host code only; the device path (scl_write_frame) copies
// the state into pinned memory and calls write_frame_files on a host thread.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "scl_frames.h"

namespace scl {

std::string fortran_e(double v, int w, int d) {
  std::string body;
  if (std::isnan(v)) {
    body = "NaN";
  } else if (std::isinf(v)) {
    body = v < 0 ? "-Infinity" : "Infinity";
  } else {
    std::string digits(d, '0');
    int e = 0;
    if (v != 0.0) {
      // d significant digits, rounded to nearest: x.xxxxe+yy -> 0.xxxxx * 10^(yy+1)
      char buf[64];
      std::snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(v));
      digits.clear();
      const char* p = buf;
      for (; *p && *p != 'e'; ++p)
        if (*p >= '0' && *p <= '9') digits.push_back(*p);
      e = std::atoi(p + 1) + 1;
    }
    body = (std::signbit(v) ? "-0." : "0.") + digits;
    char ex[8];
    const int ae = e < 0 ? -e : e;
    if (ae <= 99) std::snprintf(ex, sizeof(ex), "E%c%02d", e < 0 ? '-' : '+', ae);
    else if (ae <= 999) std::snprintf(ex, sizeof(ex), "%c%03d", e < 0 ? '-' : '+', ae);
    else return std::string(w, '*');
    body += ex;
  }
  if ((int)body.size() > w) return std::string(w, '*');
  return std::string(w - body.size(), ' ') + body;
}

namespace {

std::string i5(int v) {
  char b[32];
  std::snprintf(b, sizeof(b), "%5d", v);
  return b;
}

// out1.f90:34-42 / out2.f90:29-37: the last four digits of iframe
std::string frame_name(const std::string& dir, char kind, int iframe) {
  char b[16];
  std::snprintf(b, sizeof(b), "fort.%c%04d", kind, iframe % 10000);
  return dir.empty() ? std::string(b) : dir + "/" + b;
}

// values below 1d-99 in magnitude are written as 0 (out1.f90:62-66)
double clip(double v) { return std::fabs(v) < 1e-99 ? 0.0 : v; }

// (v(1..n)) under format (4ew.d): four values per record
void put_values(std::string& o, const double* v, int n, int w, int d) {
  for (int k = 0; k < n; ++k) {
    o += fortran_e(clip(v[k]), w, d);
    if (k % 4 == 3 || k == n - 1) o += '\n';
  }
}

// list-directed write(u,*) ' ': a leading blank, then the blank string
const char* kBlankRecord = "  \n";

std::string grid_header(const FrameSpec& f) {
  std::string o;
  o += i5(1) + "                 grid_number\n";
  o += i5(1) + "                 AMR_level\n";
  o += i5(f.mx) + "                 mx\n";
  if (f.ndim == 2) {
    o += i5(f.my) + "                 my\n";
    o += fortran_e(f.xlower, 26, 16) + "    xlow\n";
    o += fortran_e(f.ylower, 26, 16) + "    ylow\n";
    o += fortran_e(f.dx, 26, 16) + "    dx\n";
    o += fortran_e(f.dy, 26, 16) + "    dy\n\n";
  } else {
    o += fortran_e(f.xlower, 18, 8) + "    xlow\n";
    o += fortran_e(f.dx, 18, 8) + "    dx\n\n";
  }
  return o;
}

// the grid file body: out1.f90:59-72 (1-D, 4e16.8) / out2.f90:55-69 (2-D, 4e26.16)
std::string grid_body(const FrameSpec& f, const double* a, int ncomp, bool blank_after_1d_twice) {
  std::string o;
  const long ld = f.mx + 2L * f.mbc;
  const long rows = f.ndim == 2 ? f.my + 2L * f.mbc : 1;
  const long plane = ld * rows;
  double v[64];
  if (f.ndim == 1) {
    for (int i = 1; i <= f.mx; ++i) {
      for (int m = 0; m < ncomp; ++m) v[m] = a[(i + f.mbc - 1) + m * plane];
      put_values(o, v, ncomp, 16, 8);
    }
    o += kBlankRecord;
    if (blank_after_1d_twice) o += kBlankRecord;
  } else {
    for (int j = 1; j <= f.my; ++j) {
      for (int i = 1; i <= f.mx; ++i) {
        for (int m = 0; m < ncomp; ++m) v[m] = a[(i + f.mbc - 1) + (long)(j + f.mbc - 1) * ld + m * plane];
        put_values(o, v, ncomp, 26, 16);
      }
      o += kBlankRecord;
    }
    o += kBlankRecord;
  }
  return o;
}

int put_file(const std::string& path, const std::string& body, std::string* err) {
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) {
    *err = "cannot open " + path + ": " + std::strerror(errno);
    return -1;
  }
  const size_t n = std::fwrite(body.data(), 1, body.size(), fp);
  const int rc = std::fclose(fp);
  if (n != body.size() || rc != 0) {
    *err = "cannot write " + path;
    return -1;
  }
  return 0;
}

}  // namespace

int write_frame_files(const FrameSpec& f, const double* q, const double* aux, std::string* err) {
  if (f.meqn > 64 || f.maux > 64) {
    *err = "frame output supports at most 64 components";
    return -1;
  }
  std::string qf = grid_header(f) + grid_body(f, q, f.meqn, true);
  if (put_file(frame_name(f.dir, 'q', f.iframe), qf, err)) return -1;
  if (f.write_aux && aux && f.maux > 0) {
    std::string af = grid_header(f) + grid_body(f, aux, f.maux, false);
    if (put_file(frame_name(f.dir, 'a', f.iframe), af, err)) return -1;
  }
  // out1.f90:94-101 / out2.f90:107-113
  std::string tf = fortran_e(f.t, 26, 16) + "    time\n";
  tf += i5(f.meqn) + "                 meqn\n";
  tf += i5(1) + "                 ngrids\n";
  tf += i5(f.maux) + "                 maux\n";
  tf += i5(f.ndim) + "                 ndim\n\n\n";
  return put_file(frame_name(f.dir, 't', f.iframe), tf, err);
}

}  // namespace scl
