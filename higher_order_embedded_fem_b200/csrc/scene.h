// Synthetic scene data (host).
#pragma once

#include <stdint.h>

#include <vector>

#include "internal.h"

namespace hoefem {

struct SceneBlock {
  int kind = 0, nn = 0;
  std::vector<int64_t> conn;
  bool uniform = true;
  std::vector<int64_t> qoff;
  std::vector<double> qw, qp;
};

struct Scene {
  std::vector<double> X;
  std::vector<SceneBlock> blocks;
  double cell_size = 0.0;
};

Scene* scene_tet10_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cpu);
Scene* scene_hex27_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cpu);
Scene* scene_embedded_cylinder(int64_t n, double r_in, double r_out, int qmin, int qmax, uint64_t seed);
void scene_volume_fractions(const Scene& s, double* out);
void random_normal(uint64_t seed, int64_t n, double sigma, double* out);
bool tet_quadrature(int strength, std::vector<double>& w, std::vector<double>& p);
void hex_quadrature_5(std::vector<double>& w, std::vector<double>& p);

}  // namespace hoefem
