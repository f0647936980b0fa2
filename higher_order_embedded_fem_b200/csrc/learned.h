// Learned coarse correction (internal declarations).
#pragma once

#include <functional>

#include "internal.h"
#include "solver.h"

namespace hoefem {

struct Learned {
  // sizes: S coarse subdomains, NM local modes, NG global modes, F = NM + NG + 3
  // features, MLP F -> H -> H -> NM
  static constexpr int NM = 32, NG = 29, F = 64, H = 256;
  Model* m = nullptr;
  int S = 256;
  std::vector<unsigned char> bc;  // dof mask
  // partition (host) and coarse modes
  std::vector<int> sub_off;   // S + 1, offsets into sub_dofs
  std::vector<int> sub_dofs;  // dof indices grouped by subdomain
  std::vector<float> centroid;  // S x 3 (normalised to the model's bounding box)
  DBuf<int> d_sub_off, d_sub_dofs;
  DBuf<float> d_phi;        // local modes: for subdomain s, NM x n_s (row-major) at 32 * sub_off[s]
  DBuf<float> d_psi;        // global modes: NG x ndof
  DBuf<float> d_centroid;
  DBuf<float> d_gproj;      // NG global projections of the current residual
  DBuf<double> d_gpart;     // their per-chunk partial sums
  // MLP (FP32 master weights, Adam moments); layout: W1 F x H, b1 H, W2 H x H, b2 H, W3 H x NM, b3 NM
  size_t n_params = 0;
  DBuf<float> params, grads, adam_m, adam_v;
  // per-column standardisation of features and targets (statistics of the
  // training set at the last train() call); the network works on standardised
  // values, predictions are mapped back with t_mean + t_std * y
  DBuf<float> x_mean, x_std, t_mean, t_std;
  DBuf<uint16_t> params_bf16;   // BF16 copies of W1, W2, W3 for tensor-core inference
  int adam_t = 0;
  // activations (batch up to max_batch rows)
  int max_batch = 0;
  DBuf<float> X, Y1, Y2, Y3, T, dY1, dY2, dY3;
  // dataset
  DBuf<float> data_X, data_T;
  long long n_data = 0, cap_data = 0;
  // scratch
  DBuf<double> e, rtmp, partials, scal;
  DBuf<unsigned> counter;
  double* h_scal = nullptr;
  bool trained = false;
  int use_bf16 = 1;
  ~Learned();

  void setup(Model* model, const unsigned char* bc_mask, int num_sub, uint64_t seed);
  // features of residual r (device, FP64) into X rows [row0, row0 + S); returns ||r||
  double features(const double* r, float* Xout, cudaStream_t s);
  // x0 = ||r|| * sum_s Phi_s c_s from coefficients C (S x NM)
  void apply(const float* C, double rnorm, double* x0, cudaStream_t s);
  // coarse coefficients of a correction e: T rows = Phi_s e_s / rnorm
  void targets(const double* e, double rnorm, float* Tout, cudaStream_t s);
  void add_pair(const double* r, const double* e, cudaStream_t s);
  void forward(const float* Xin, int rows, bool bf16, cudaStream_t s);  // -> Y3
  float train_step(const float* Xb, const float* Tb, int rows, float lr, cudaStream_t s);  // returns loss
  void refresh_bf16(cudaStream_t s);
  void train(long long steps, int batch, float lr, uint64_t seed, float* loss_hist, cudaStream_t s);
  // prediction for residual r: writes x0 (device FP64)
  void predict(const double* r, double* x0, cudaStream_t s);
  // the same without a host round trip (graph-capturable): ||r|| = sqrt(*rr)
  // read on the device
  void predict_device(const double* r, const double* rr, double* x0, cudaStream_t s);
};

}  // namespace hoefem
