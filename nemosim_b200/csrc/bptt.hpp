// bptt.hpp -- the differentiable float32 mode (see bptt.cu for the model).
#pragma once

#include <stddef.h>

#include <vector>

namespace nemo_b200 {

struct BpttDev {
	int N, B, T, R, ckpt, smooth;
	float alpha, lossScale;
	const int* inStart;   // [N+1] in-synapses by target
	const int* inSrc;
	const int* inDelay;
	const int* inSyn;     // synapse index (into W)
	const int* outStart;  // [N+1] out-synapses by source (synapse index = position)
	const int* outTgt;
	const int* outDelay;
	float* S;             // [N][T][B]
	float* v;             // [N][B]
	float* u;
	float* ckV;           // [nck][N][B]
	float* ckU;
	float* r;             // [R][B]
	float* rHist;         // [R][T][B]
	float* lossPart;      // [N][B]
	float* segV;          // [ckpt][N][B]
	float* segU;
	float* segSyn;
	float* lamV;          // [N][B]
	float* lamU;
	float* lamR;          // [R][B]
	float* lamI;          // [N][T][B]
	float* gA;            // [N][B]
	float* gB;
};

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
	// M synapses, ordered by source; synapse e has weight W[e]
	Bptt(unsigned N, unsigned B, unsigned T, unsigned R, unsigned ckpt, size_t M, const unsigned* src,
			const unsigned* tgt, const unsigned* delay, int smooth, int device);
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
	int m_device = 0;
	size_t m_M = 0;
	std::vector<void*> m_allocs;
	float* alloc(size_t n);
	const int* upload(const std::vector<int>& v);
};

} // namespace nemo_b200
