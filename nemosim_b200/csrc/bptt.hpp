// bptt.hpp -- the differentiable mode (see bptt.cu for the model).
#pragma once

#include <stddef.h>

#include <vector>

namespace nemo_b200 {

// sizes and synapse structure (shared by both state types)
struct BpttDev {
	int N, B, T, R, ckpt, smooth;
	const int* inStart;   // [N+1] in-synapses by target
	const int* inSrc;
	const int* inDelay;
	const int* inSyn;     // synapse index (into W)
	const int* outStart;  // [N+1] out-synapses by source (synapse index = position)
	const int* outTgt;
	const int* outDelay;
};

// state, trajectory and adjoint arrays in the state type Real
template<typename Real>
struct BpttState {
	Real alpha, lossScale;
	Real* S;              // [N][T][B]
	Real* v;              // [N][B]
	Real* u;
	Real* ckV;            // [nck][N][B]
	Real* ckU;
	Real* r;              // [R][B]
	Real* rHist;          // [R][T][B]
	Real* lossPart;       // [N][B]
	Real* segV;           // [ckpt][N][B]
	Real* segU;
	Real* segSyn;
	Real* lamV;           // [N][B]
	Real* lamU;
	Real* lamR;           // [R][B]
	Real* lamI;           // [N][T][B]
	Real* gA;             // [N][B]
	Real* gB;
};

// the caller's float32 tensors (device pointers)
struct BpttParams {
	const float* W;
	const float* a;
	const float* b;
	const float* c;
	const float* d;
	const float* noise;   // [T][B][N]
	const float* target;  // [T][B][R]
};

class Bptt {
public:
	// M synapses, ordered by source; synapse e has weight W[e].  smooth:
	// fast sigmoid in the forward pass; fp64: neuron state, trajectories and
	// adjoints in float64 (inputs and gradients stay float32).
	Bptt(unsigned N, unsigned B, unsigned T, unsigned R, unsigned ckpt, size_t M, const unsigned* src,
			const unsigned* tgt, const unsigned* delay, bool smooth, bool fp64, int device);
	~Bptt();
	// forward pass; *loss (device) receives the loss
	void forward(const BpttParams& P, float* loss, void* stream);
	// gradients of the loss of the last forward pass (device arrays)
	void backward(const BpttParams& P, float* dW, float* da, float* db, void* stream);
	// filtered readout spike trains of the last forward pass, [T][B][R]
	void readout(float* out, void* stream);
	size_t synapses() const { return m_M; }
	unsigned neurons() const { return (unsigned) D.N; }

private:
	BpttDev D;
	bool m_fp64 = false;
	BpttState<float> X32{};
	BpttState<double> X64{};
	int m_device = 0;
	size_t m_M = 0;
	std::vector<void*> m_allocs;
	void* alloc(size_t bytes);
	const int* upload(const std::vector<int>& v);
	template<typename Real> void allocState(BpttState<Real>& X);
	template<typename Real> void forwardT(BpttState<Real>& X, const BpttParams& P, float* loss, void* stream);
	template<typename Real> void backwardT(BpttState<Real>& X, const BpttParams& P, float* dW, float* da,
			float* db, void* stream);
	template<typename Real> void readoutT(BpttState<Real>& X, float* out, void* stream);
};

} // namespace nemo_b200
