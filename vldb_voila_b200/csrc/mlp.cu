/*
 * The learned flavor chooser's network: a 3-layer perceptron (in -> hidden -> hidden -> out,
 * ReLU) trained and evaluated on the GPU by hand-written kernels.  The reference searches
 * the blend space by running variants (explorer.cpp:111-134, :352-426); here a network maps
 * per-pipeline features to the predicted relative time of each candidate flavor, trained on
 * timings measured by the exhaustive autotuner, which stays its fallback and yardstick.
 *
 * Sizes are tiny (tens of features, a few dozen flavors, <= a few thousand samples), so the
 * layers are plain FFMA kernels: one thread per output element, fp32, deterministic (no
 * atomics; reductions run in a fixed order).
 *
 * Loss: masked mean squared error over the outputs, sum(mask * (y - t)^2) / sum(mask).
 * Optimiser: Adam (Kingma & Ba 2015) with bias correction.
 */
#include <cmath>
#include <functional>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "engine_internal.hpp"

namespace vc {

/* ------------------------------------------------------------------ kernels ------------ */

/* Y[n][o] = act(sum_i X[n][i] * W[i][o] + b[o]) */
__global__ void mlp_linear_fwd(const float* __restrict__ X, const float* __restrict__ W, const float* __restrict__ b,
	float* __restrict__ Y, int N, int I, int O, int relu)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= N * O) {
		return;
	}
	const int n = idx / O, o = idx % O;
	float acc = b[o];
	for (int i = 0; i < I; i++) {
		acc = fmaf(X[n * I + i], W[i * O + o], acc);
	}
	Y[idx] = relu && acc < 0.f ? 0.f : acc;
}

/* dX[n][i] = (sum_o dY[n][o] * W[i][o]) * (Xact[n][i] > 0)  (ReLU derivative of the input) */
__global__ void mlp_linear_bwd_input(const float* __restrict__ dY, const float* __restrict__ W,
	const float* __restrict__ Xact, float* __restrict__ dX, int N, int I, int O)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= N * I) {
		return;
	}
	const int n = idx / I, i = idx % I;
	float acc = 0.f;
	for (int o = 0; o < O; o++) {
		acc = fmaf(dY[n * O + o], W[i * O + o], acc);
	}
	dX[idx] = Xact[idx] > 0.f ? acc : 0.f;
}

/* dW[i][o] = sum_n X[n][i] * dY[n][o];  db[o] = sum_n dY[n][o] (threads i == I compute db) */
__global__ void mlp_linear_bwd_weight(const float* __restrict__ X, const float* __restrict__ dY,
	float* __restrict__ dW, float* __restrict__ db, int N, int I, int O)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (I + 1) * O) {
		return;
	}
	const int i = idx / O, o = idx % O;
	float acc = 0.f;
	if (i < I) {
		for (int n = 0; n < N; n++) {
			acc = fmaf(X[n * I + i], dY[n * O + o], acc);
		}
		dW[i * O + o] = acc;
	} else {
		for (int n = 0; n < N; n++) {
			acc += dY[n * O + o];
		}
		db[o] = acc;
	}
}

/* dY = 2 * mask * (Y - T) / sum(mask); loss (one block) */
__global__ void mlp_loss_grad(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ M,
	float* __restrict__ dY, float* __restrict__ loss, int total)
{
	__shared__ float s_err[256];
	__shared__ float s_cnt[256];
	float e = 0.f, c = 0.f;
	for (int i = threadIdx.x; i < total; i += blockDim.x) {
		const float d = Y[i] - T[i];
		e += M[i] * d * d;
		c += M[i];
	}
	s_err[threadIdx.x] = e;
	s_cnt[threadIdx.x] = c;
	__syncthreads();
	for (int s = blockDim.x / 2; s > 0; s >>= 1) {
		if ((int)threadIdx.x < s) {
			s_err[threadIdx.x] += s_err[threadIdx.x + s];
			s_cnt[threadIdx.x] += s_cnt[threadIdx.x + s];
		}
		__syncthreads();
	}
	const float denom = s_cnt[0] > 0.f ? s_cnt[0] : 1.f;
	for (int i = threadIdx.x; i < total; i += blockDim.x) {
		dY[i] = 2.f * M[i] * (Y[i] - T[i]) / denom;
	}
	if (threadIdx.x == 0) {
		*loss = s_err[0] / denom;
	}
}

__global__ void mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
	int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) {
		return;
	}
	const float gi = g[i];
	const float mi = b1 * m[i] + (1.f - b1) * gi;
	const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
	m[i] = mi;
	v[i] = vi;
	p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

/* ------------------------------------------------------------------ host side ---------- */

struct Mlp {
	int device = 0;
	int in = 0, hid = 0, out = 0;
	int64_t nparams = 0;
	float* params = nullptr; /* W1 b1 W2 b2 W3 b3 */
	float* grads = nullptr;
	float* m = nullptr;
	float* v = nullptr;
	int64_t step = 0;
	int cap = 0;             /* activation buffers sized for this many samples */
	float *X = nullptr, *T = nullptr, *M = nullptr, *H1 = nullptr, *H2 = nullptr, *Y = nullptr;
	float *dY = nullptr, *dH2 = nullptr, *dH1 = nullptr, *loss = nullptr;

	int64_t off_W1() const { return 0; }
	int64_t off_b1() const { return off_W1() + (int64_t)in * hid; }
	int64_t off_W2() const { return off_b1() + hid; }
	int64_t off_b2() const { return off_W2() + (int64_t)hid * hid; }
	int64_t off_W3() const { return off_b2() + hid; }
	int64_t off_b3() const { return off_W3() + (int64_t)hid * out; }

	void free_acts() {
		for (float* p : {X, T, M, H1, H2, Y, dY, dH2, dH1}) {
			if (p) {
				cudaFree(p);
			}
		}
		X = T = M = H1 = H2 = Y = dY = dH2 = dH1 = nullptr;
		cap = 0;
	}

	void ensure(int n) {
		if (n <= cap) {
			return;
		}
		free_acts();
		cap = n;
		VC_CHECK_CUDA(cudaMalloc(&X, sizeof(float) * (size_t)n * in));
		VC_CHECK_CUDA(cudaMalloc(&T, sizeof(float) * (size_t)n * out));
		VC_CHECK_CUDA(cudaMalloc(&M, sizeof(float) * (size_t)n * out));
		VC_CHECK_CUDA(cudaMalloc(&H1, sizeof(float) * (size_t)n * hid));
		VC_CHECK_CUDA(cudaMalloc(&H2, sizeof(float) * (size_t)n * hid));
		VC_CHECK_CUDA(cudaMalloc(&Y, sizeof(float) * (size_t)n * out));
		VC_CHECK_CUDA(cudaMalloc(&dY, sizeof(float) * (size_t)n * out));
		VC_CHECK_CUDA(cudaMalloc(&dH2, sizeof(float) * (size_t)n * hid));
		VC_CHECK_CUDA(cudaMalloc(&dH1, sizeof(float) * (size_t)n * hid));
	}

	~Mlp() {
		cudaSetDevice(device);
		free_acts();
		for (float* p : {params, grads, m, v, loss}) {
			if (p) {
				cudaFree(p);
			}
		}
	}

	static unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

	void forward(int n) {
		mlp_linear_fwd<<<blocks((int64_t)n * hid), 256>>>(X, params + off_W1(), params + off_b1(), H1, n, in, hid, 1);
		mlp_linear_fwd<<<blocks((int64_t)n * hid), 256>>>(H1, params + off_W2(), params + off_b2(), H2, n, hid, hid, 1);
		mlp_linear_fwd<<<blocks((int64_t)n * out), 256>>>(H2, params + off_W3(), params + off_b3(), Y, n, hid, out, 0);
	}

	void backward(int n) {
		mlp_loss_grad<<<1, 256>>>(Y, T, M, dY, loss, n * out);
		mlp_linear_bwd_weight<<<blocks((int64_t)(hid + 1) * out), 256>>>(H2, dY, grads + off_W3(), grads + off_b3(), n,
			hid, out);
		mlp_linear_bwd_input<<<blocks((int64_t)n * hid), 256>>>(dY, params + off_W3(), H2, dH2, n, hid, out);
		mlp_linear_bwd_weight<<<blocks((int64_t)(hid + 1) * hid), 256>>>(H1, dH2, grads + off_W2(), grads + off_b2(), n,
			hid, hid);
		mlp_linear_bwd_input<<<blocks((int64_t)n * hid), 256>>>(dH2, params + off_W2(), H1, dH1, n, hid, hid);
		mlp_linear_bwd_weight<<<blocks((int64_t)(in + 1) * hid), 256>>>(X, dH1, grads + off_W1(), grads + off_b1(), n,
			in, hid);
	}

	void adam(float lr) {
		step++;
		const float b1 = 0.9f, b2 = 0.999f;
		const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
		mlp_adam<<<blocks(nparams), 256>>>(params, grads, m, v, (int)nparams, lr, b1, b2, 1e-8f, c1, c2);
	}
};

} // namespace vc

/* ====================================================================== C ABI ======== */

#include "../../include/voila_cuda.h"

using vc::Error;
using vc::Mlp;

struct vc_mlp {
	Mlp m;
};

namespace vc {
int abi_guard_mlp(const std::function<void()>& f);
}

extern "C" {

int vc_mlp_create(int device, int n_in, int n_hidden, int n_out, uint64_t seed, vc_mlp** out)
{
	return vc::abi_guard_mlp([&] {
		if (!out || n_in < 1 || n_hidden < 1 || n_out < 1 || n_in > 4096 || n_hidden > 4096 || n_out > 4096) {
			throw Error(VC_ERR_INVALID, "bad network shape");
		}
		int ndev = 0;
		if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
			cudaGetLastError();
			throw Error(VC_ERR_NO_DEVICE, "no CUDA device is available");
		}
		VC_CHECK_CUDA(cudaSetDevice(device));
		auto* h = new vc_mlp();
		Mlp& m = h->m;
		m.device = device;
		m.in = n_in;
		m.hid = n_hidden;
		m.out = n_out;
		m.nparams = m.off_b3() + n_out;
		std::vector<float> init((size_t)m.nparams, 0.f);
		/* Glorot-uniform weights from a seeded SplitMix64 stream, zero biases */
		uint64_t s = seed;
		auto uni = [&]() {
			s += 0x9e3779b97f4a7c15ull;
			uint64_t z = s;
			z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
			z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
			z ^= z >> 31;
			return (double)(z >> 11) * (1.0 / 9007199254740992.0);
		};
		auto fill = [&](int64_t off, int fan_in, int fan_out) {
			const double lim = std::sqrt(6.0 / (fan_in + fan_out));
			for (int64_t i = 0; i < (int64_t)fan_in * fan_out; i++) {
				init[(size_t)(off + i)] = (float)((2.0 * uni() - 1.0) * lim);
			}
		};
		fill(m.off_W1(), n_in, n_hidden);
		fill(m.off_W2(), n_hidden, n_hidden);
		fill(m.off_W3(), n_hidden, n_out);
		const size_t bytes = sizeof(float) * (size_t)m.nparams;
		try {
			VC_CHECK_CUDA(cudaMalloc(&m.params, bytes));
			VC_CHECK_CUDA(cudaMalloc(&m.grads, bytes));
			VC_CHECK_CUDA(cudaMalloc(&m.m, bytes));
			VC_CHECK_CUDA(cudaMalloc(&m.v, bytes));
			VC_CHECK_CUDA(cudaMalloc(&m.loss, sizeof(float)));
			VC_CHECK_CUDA(cudaMemcpy(m.params, init.data(), bytes, cudaMemcpyHostToDevice));
			VC_CHECK_CUDA(cudaMemset(m.grads, 0, bytes));
			VC_CHECK_CUDA(cudaMemset(m.m, 0, bytes));
			VC_CHECK_CUDA(cudaMemset(m.v, 0, bytes));
		} catch (...) {
			delete h;
			throw;
		}
		*out = h;
	});
}

int vc_mlp_free(vc_mlp* h)
{
	return vc::abi_guard_mlp([&] { delete h; });
}

int vc_mlp_num_params(vc_mlp* h, int64_t* n)
{
	return vc::abi_guard_mlp([&] {
		if (!h || !n) {
			throw Error(VC_ERR_INVALID, "null argument");
		}
		*n = h->m.nparams;
	});
}

int vc_mlp_get_params(vc_mlp* h, float* out, int64_t cap)
{
	return vc::abi_guard_mlp([&] {
		if (!h || !out || cap < h->m.nparams) {
			throw Error(VC_ERR_INVALID, "parameter buffer too small");
		}
		VC_CHECK_CUDA(cudaSetDevice(h->m.device));
		VC_CHECK_CUDA(cudaMemcpy(out, h->m.params, sizeof(float) * (size_t)h->m.nparams, cudaMemcpyDeviceToHost));
	});
}

int vc_mlp_set_params(vc_mlp* h, const float* in, int64_t n)
{
	return vc::abi_guard_mlp([&] {
		if (!h || !in || n != h->m.nparams) {
			throw Error(VC_ERR_INVALID, "parameter count mismatch");
		}
		VC_CHECK_CUDA(cudaSetDevice(h->m.device));
		VC_CHECK_CUDA(cudaMemcpy(h->m.params, in, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice));
	});
}

static void upload_batch(Mlp& m, const float* X, const float* T, const float* M, int n)
{
	m.ensure(n);
	VC_CHECK_CUDA(cudaMemcpy(m.X, X, sizeof(float) * (size_t)n * m.in, cudaMemcpyHostToDevice));
	if (T) {
		VC_CHECK_CUDA(cudaMemcpy(m.T, T, sizeof(float) * (size_t)n * m.out, cudaMemcpyHostToDevice));
	}
	if (T) {
		if (M) {
			VC_CHECK_CUDA(cudaMemcpy(m.M, M, sizeof(float) * (size_t)n * m.out, cudaMemcpyHostToDevice));
		} else {
			std::vector<float> ones((size_t)n * m.out, 1.f);
			VC_CHECK_CUDA(cudaMemcpy(m.M, ones.data(), sizeof(float) * ones.size(), cudaMemcpyHostToDevice));
		}
	}
}

int vc_mlp_loss_grad(vc_mlp* h, const float* X, const float* T, const float* M, int n, float* loss, float* grads)
{
	return vc::abi_guard_mlp([&] {
		if (!h || !X || !T || n < 1) {
			throw Error(VC_ERR_INVALID, "bad arguments");
		}
		Mlp& m = h->m;
		VC_CHECK_CUDA(cudaSetDevice(m.device));
		upload_batch(m, X, T, M, n);
		m.forward(n);
		m.backward(n);
		VC_CHECK_CUDA(cudaGetLastError());
		if (loss) {
			VC_CHECK_CUDA(cudaMemcpy(loss, m.loss, sizeof(float), cudaMemcpyDeviceToHost));
		}
		if (grads) {
			VC_CHECK_CUDA(cudaMemcpy(grads, m.grads, sizeof(float) * (size_t)m.nparams, cudaMemcpyDeviceToHost));
		}
	});
}

int vc_mlp_train(vc_mlp* h, const float* X, const float* T, const float* M, int n, int epochs, int batch, float lr,
	uint64_t seed, float* final_loss)
{
	return vc::abi_guard_mlp([&] {
		if (!h || !X || !T || n < 1 || epochs < 0 || batch < 1 || !(lr > 0.f)) {
			throw Error(VC_ERR_INVALID, "bad arguments");
		}
		Mlp& m = h->m;
		VC_CHECK_CUDA(cudaSetDevice(m.device));
		if (batch > n) {
			batch = n;
		}
		std::vector<int> order((size_t)n);
		for (int i = 0; i < n; i++) {
			order[(size_t)i] = i;
		}
		std::vector<float> bx((size_t)batch * m.in), bt((size_t)batch * m.out), bm((size_t)batch * m.out);
		uint64_t s = seed;
		auto next = [&]() {
			s += 0x9e3779b97f4a7c15ull;
			uint64_t z = s;
			z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
			z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
			return z ^ (z >> 31);
		};
		float last = 0.f;
		for (int e = 0; e < epochs; e++) {
			for (int i = n - 1; i > 0; i--) { /* Fisher-Yates shuffle per epoch */
				std::swap(order[(size_t)i], order[(size_t)(next() % (uint64_t)(i + 1))]);
			}
			for (int b0 = 0; b0 < n; b0 += batch) {
				const int nb = std::min(batch, n - b0);
				for (int r = 0; r < nb; r++) {
					const int src = order[(size_t)(b0 + r)];
					std::memcpy(&bx[(size_t)r * m.in], X + (size_t)src * m.in, sizeof(float) * m.in);
					std::memcpy(&bt[(size_t)r * m.out], T + (size_t)src * m.out, sizeof(float) * m.out);
					for (int o = 0; o < m.out; o++) {
						bm[(size_t)r * m.out + o] = M ? M[(size_t)src * m.out + o] : 1.f;
					}
				}
				upload_batch(m, bx.data(), bt.data(), bm.data(), nb);
				m.forward(nb);
				m.backward(nb);
				m.adam(lr);
			}
		}
		VC_CHECK_CUDA(cudaGetLastError());
		/* loss over the whole training set */
		upload_batch(m, X, T, M, n);
		m.forward(n);
		vc::mlp_loss_grad<<<1, 256>>>(m.Y, m.T, m.M, m.dY, m.loss, n * m.out);
		VC_CHECK_CUDA(cudaMemcpy(&last, m.loss, sizeof(float), cudaMemcpyDeviceToHost));
		if (final_loss) {
			*final_loss = last;
		}
	});
}

int vc_mlp_predict(vc_mlp* h, const float* X, int n, float* Y)
{
	return vc::abi_guard_mlp([&] {
		if (!h || !X || !Y || n < 1) {
			throw Error(VC_ERR_INVALID, "bad arguments");
		}
		Mlp& m = h->m;
		VC_CHECK_CUDA(cudaSetDevice(m.device));
		upload_batch(m, X, nullptr, nullptr, n);
		m.forward(n);
		VC_CHECK_CUDA(cudaGetLastError());
		VC_CHECK_CUDA(cudaMemcpy(Y, m.Y, sizeof(float) * (size_t)n * m.out, cudaMemcpyDeviceToHost));
	});
}

} // extern "C"
