// warmstart.cuh -- host-side state of the learned warm-start network
// (kernels and the description of the network in warmstart.cu).
#pragma once

#include <cuda_bf16.h>

#include <memory>
#include <vector>

#include "tabi_impl.cuh"

namespace tabi {

constexpr int kWsK = 16;  // neighbours per panel
constexpr int kWsR = 8;   // radial basis functions of the edge input
constexpr int kWsF = 10;  // node input features

// One molecule's panels: FP64 components with a stride (3 for the reference's
// interleaved tr_xyz / tr_q, 1 for the handle's SoA arrays), area (n), the
// right-hand side b (2n) and, optionally, z = M^-1 b (2n), the leaf-block
// preconditioner's solution, which the network takes as input and corrects.
struct WsInput {
  int n = 0;
  const double *px = nullptr, *py = nullptr, *pz = nullptr;
  int ps = 1;
  const double *qx = nullptr, *qy = nullptr, *qz = nullptr;
  int qs = 1;
  const double* area = nullptr;
  const double* b = nullptr;
  const double* z = nullptr;  // may be null: the baseline is then [0; b2]
};

struct WsNet {
  WsNet(int hidden, int layers, unsigned long long seed);
  ~WsNet();
  WsNet(const WsNet&) = delete;
  WsNet& operator=(const WsNet&) = delete;

  int H, L;
  int64_t np = 0;
  struct Layer {
    int64_t Wa, Wf, bf, Wb1, Wb2, bb;
  };
  int64_t off_W0 = 0, off_b0 = 0, off_Wo = 0, off_bo = 0;
  std::vector<Layer> lay;
  int64_t adam_t = 0;
  cudaStream_t stream = nullptr;
  double* h_stats = nullptr;  // pinned

  DBuf<float> theta, grad, m, v;
  DBuf<__nv_bfloat16> wbf;
  // per-molecule state (grow-only)
  DBuf<float4> pos, nrm;
  DBuf<float2> bfl, zfl;
  DBuf<double> stats_part, stats;
  DBuf<int> cell, ccnt, coff, csorted, sbuf, nbr, err, rcnt, roff, rev;
  DBuf<float> dbar, feat;
  DBuf<float> hs, us, as, zs, pre0, dout;
  DBuf<double> lpart;
  DBuf<float> dh, dz, da, du, part, part2, wpart;

  // a second network with the same parameters (own buffers and stream)
  std::unique_ptr<WsNet> clone() const;
  void set_params(const float* th);
  void get_params(float* th);
  // neighbour graph and node features of a molecule
  void graph(const WsInput& in, cudaStream_t s);
  // forward pass; xout (2n, may be null) gets the prediction, target (2n,
  // may be null) makes it compute the loss and its output gradient
  void forward(const WsInput& in, double* xout, const double* target, cudaStream_t s);
  // gradients of the last forward-with-target into grad
  void backward(int n, cudaStream_t s);
  void adam(double lr, cudaStream_t s);
  double read_loss(cudaStream_t s);
  bool graph_exact(cudaStream_t s);

 private:
  void dw(int M, int Kd, int N, const float* A, const float* D, float* g, cudaStream_t s);
  void colsum(int M, int N, const float* X, float* g, cudaStream_t s);
};

}  // namespace tabi
