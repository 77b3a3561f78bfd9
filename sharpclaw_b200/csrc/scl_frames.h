// scl_frames.h -- frame files in the format of src/1d/out1.f90 and
// src/2d/out2.f90 (fort.qNNNN, fort.tNNNN, fort.aNNNN), host code.
#pragma once
#include <string>

namespace scl {

// Everything a frame file records besides the arrays.
struct FrameSpec {
  int ndim, mx, my, mbc, meqn, maux;
  double xlower, ylower, dx, dy;
  double t;
  int iframe;
  bool write_aux;
  std::string dir;
};

// Fortran Ew.d output as gfortran writes it: [-]0.<d digits>E+xx, or +xxx
// for a three-digit exponent, right-justified in w columns.
std::string fortran_e(double v, int w, int d);

// Writes the frame files from host arrays in the reference layout (double,
// ghost cells included).  Returns 0, or -1 with *err set.
int write_frame_files(const FrameSpec& f, const double* q, const double* aux, std::string* err);

}  // namespace scl
