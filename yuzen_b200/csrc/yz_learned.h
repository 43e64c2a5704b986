// yz_learned.h -- the learned preconditioner: a small U-Net on the film's
// grid, BF16 3x3 convolutions on the tensor cores (tcgen05, FP32
// accumulation in TMEM), trained on the device from the (residual, matrix
// diagonal, film height) -> AMG-correction pairs the solver generates.
//
// The network maps a residual r (a vector over the n = nx*ny rows of the
// ghost-padded grid) to z = N(r) ~ M r, where M is the SA-AMG V-cycle the
// solver would apply.  Its input channels are r / rms(r) and its products with two
// feature maps of the system -- f1 = log10 |a_ii| / 4 of the unscaled
// matrix's diagonal, f2 = log10 h / 2 + 1 of the film height (0 where the
// caller gives none) -- namely r, r f1, r f2, r f1^2, r f2^2, r f1 f2; the
// output, scaled back by rms(r), is z.  Every input channel is linear in r:
// with the activation off (the preconditioner's form) the network has no
// bias and no ReLU and is a linear operator on r whose coefficients vary
// with f1 and f2, so BiCGStab sees one fixed preconditioner per system; with
// ReLU on it is the usual nonlinear U-Net.  Architecture (channels per level
// 16, 32, 64, 64; every convolution 3x3):
//
//   F(16: 3 used) -enc0-> E0(16) -pool-> P1 -enc1-> E1(32) -pool-> P2 -enc2->
//   E2(64) -pool-> P3 -bott-> B3(64) -up, concat E2-> dec2 -> D2(64) -up,
//   concat E1-> dec1 -> D1(32) -up, concat E0-> dec0 -> D0(16) -1x1-> z
//
// Images: level l is H_l x W_l pixels (H_0 = 8 ceil(ny/8), W_0 = 8 (ceil(nx/8)
// + 1), halved per level), row-major, channels innermost (NHWC, bf16); the
// real region of level 0 is the ny x nx grid, of level l+1 the ceil of half
// the level-l one; every activation is 0 outside it.  A 3x3 convolution
// reads pixel p + dy W + dx (zero outside the image): with at least one zero
// column right of the real region at every level, that is the convolution
// with zero padding of the real region.
#pragma once

#include "yz_common.cuh"

#include <cuda_bf16.h>
#include <vector>

namespace yz {

struct ConvLayer
{
	int cin = 0, cout = 0, level = 0;
	size_t wOff = 0, bOff = 0;      // offsets of W [cout][9][cin] and b [cout] in the parameter array
};

class Learned
{
public:
	//  capacity: training samples held on the device; seed: the weights'
	//  initialisation (He-normal from a fixed generator); act 0: linear (no
	//  bias, no activation), 1: bias and ReLU
	Learned(int device, int nx, int ny, int capacity, unsigned seed, int act);
	~Learned();

	int Nx() const { return _nx; }
	int Ny() const { return _ny; }
	int Rows() const { return _n; }
	size_t ParamCount() const { return _np; }
	int Samples() const { return _count < _cap ? _count : _cap; }
	int Capacity() const { return _cap; }
	bool Trained() const { return _trained; }

	//  the feature maps of the present system: the unscaled matrix's
	//  diagonal (values in storage order, diagonal first in each row) and the
	//  film height (null: none); queued on st
	void SetAux(const double *dValues, const int *rowptr, const double *h, cudaStream_t st);
	//  z = N(r) on the device, queued on st; with halt non-null every
	//  kernel returns at once while *halt != 0 (a finished Krylov run)
	void Apply(const double *r, double *z, cudaStream_t st, const int *halt);
	//  a training pair (r, z = M r) with the present features, stored as
	//  r / rms(r) and z / rms(r) in the next slot of the ring (queued on st;
	//  the slot is marked unused when *halt != 0 then)
	void AddSample(const double *r, const double *z, cudaStream_t st, const int *halt);
	//  the same from host arrays (n each; h may be null)
	void AddSampleHost(const double *r, const double *z, const double *diag, const double *h, cudaStream_t st);
	//  Adam on the samples held (the last `holdout` of them kept out):
	//  iters steps of `batch` samples each; returns the mean loss of the last
	//  step and, in *valErr, the relative error ||N(r) - M r|| / ||M r|| over
	//  the held-out samples (the AMG as the yardstick of the network)
	double Train(int iters, int batch, float lr, int holdout, double *valErr, cudaStream_t st);
	//  relative error over held-out samples [first, first + count)
	double Validate(int first, int count, cudaStream_t st);

	//  parameters (FP32 master copy, ParamCount values)
	void GetParams(float *out, cudaStream_t st);
	void SetParams(const float *in, cudaStream_t st);
	//  slot k of the sample ring (0 <= k < Samples()): r / rms(r), z / rms(r)
	//  and the two feature maps, n floats each; returns whether the slot holds
	//  a pair (a pair queued after its run had ended is marked unused)
	bool GetSample(int k, float *out, cudaStream_t st);
	//  one sample's loss and the gradient of it w.r.t. every parameter
	//  (features and target as normalised host maps over the n rows; the
	//  target in units of the targets' scale)
	double LossGrad(const float *feat3, const float *target, float *grad, cudaStream_t st);
	//  the network's output for host feature maps, in the units of z / rms(r)
	//  (the output layer's value times the targets' scale)
	void Forward(const float *feat3, float *out, cudaStream_t st);

private:
	struct Level { int H, W, realH, realW; };
	void Pack(cudaStream_t st);
	void ForwardImage(cudaStream_t st, const int *halt);
	void BackwardImage(cudaStream_t st);
	void Conv(const ConvLayer &L, bool transpose, const __nv_bfloat16 *x, __nv_bfloat16 *y, int ldy, int coff,
	          bool relu, cudaStream_t st, const int *halt);
	void WGrad(const ConvLayer &L, const __nv_bfloat16 *x, const __nv_bfloat16 *dy, cudaStream_t st);
	void BuildImage(int slot, cudaStream_t st);
	void Check(cudaStream_t st);

	int _device, _nx, _ny, _n;
	int _act = 0;
	Level _lv[4];
	std::vector<ConvLayer> _conv;   // enc0, enc1, enc2, bott, dec2, dec1, dec0
	size_t _np = 0, _outW = 0, _outB = 0;
	DBuf<float> _param, _grad, _m, _v;
	DBuf<__nv_bfloat16> _wf, _wb;  // packed forward / transposed weights
	std::vector<size_t> _wfOff, _wbOff;
	int _adamT = 0;
	//  activations (bf16, NHWC) and their gradients
	DBuf<__nv_bfloat16> _F, _U0, _P1, _U1, _P2, _U2, _P3, _B3, _D2, _D1, _D0;
	DBuf<__nv_bfloat16> _gD0, _gU0, _gD1, _gE0, _gU1, _gD2, _gE1, _gU2, _gB3, _gE2, _gP3, _gP2, _gP1;
	DBuf<float> _T, _part, _partB, _lossPart;
	int _partBlocks = 0;
	DBuf<double> _outSum;          // the loss and the output layer's gradient
	//  features and the Krylov vector's scale
	DBuf<float> _aux;              // [2][n]: diagonal and height features
	DBuf<double> _rms, _red;
	DBuf<unsigned int> _cnt;
	DBuf<float> _inv;              // per call: 1 / rms as float
	//  the sample ring: [cap][4][n] floats (r/rms, z/rms, diag, h features)
	DBuf<float> _ring;
	DBuf<int> _valid;
	int _cap = 0, _count = 0;
	bool _trained = false;
	DBuf<int> _err;
	//  the training targets' scale (z / rms(r) divided by it is what the
	//  network learns), set by the first training from its pairs; 1 before
	DBuf<float> _tsc;
	float _tscHost = 1.0f;
	bool _tscSet = false;
};

} // namespace yz
