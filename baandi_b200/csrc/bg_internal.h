// Internal declarations shared by the host setup, the operator runtime and the
// CUDA launchers of libbaandi_b200.so.
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/baandi_gpu.h"

namespace bg {

struct Cell {
  double lattice[3][3];  // [cart][vector]
  double recip[3][3];    // [cart][vector], B = 2 pi A^-T
  double volume;
};

struct Basis {
  int64_t npw = 0;
  std::vector<int32_t> miller;  // 3*npw
  std::vector<double> kpg;      // 3*npw
  std::vector<double> kpg2;     // npw
  double kfrac[3] = {0, 0, 0};
};

struct Species {
  double z;
  int mesh;
  const double* r;
  const double* rab;
  const double* local;
  int nbeta;
  const int32_t* l;
  const int32_t* ulen;
  const double* const* u;
  const double* dij;
  int natoms;
  const double* positions;
};

int cell_init(const double rows[9], Cell* c);
int basis_build(const Cell& cell, double ecut, const double kfrac[3], Basis* out);
int grid_dims(const Cell& cell, double ecut, int dims[3], int required[3]);
int fft_index(const int32_t* miller, int64_t npw, const int dims[3], bool gamma, int64_t* flat);
int half_sphere(const int32_t* miller, int64_t npw, std::vector<int64_t>* plus, std::vector<int64_t>* minus);
int projector_count(int nspecies, const Species* sp, int* nproj, int* natoms);
int projectors_build(double volume, int64_t npw, const double* kpg, const double* kpg2, int nspecies,
                     const Species* sp, std::complex<double>* table, int32_t* channels, double* couplings);
int local_form_factor(const Species& s, double volume, int64_t n, const double* g, double* out);
int ewald_energy(const Cell& cell, int natoms, const double* pos, const double* charge, double* out);
int atomic_charge_transform(int mesh, const double* r, const double* rab, const double* f, double volume,
                            int64_t n, const double* q, double* out);

// Thread-local message of the last failure outside a context.
void set_global_error(const std::string& msg);
std::string global_error();

}  // namespace bg
