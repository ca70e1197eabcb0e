// Far-field surrogate for ERIDA classes: a small MLP, trained on this device
// by the kernels below on exact class values that the staged contraction
// computes, predicts the residual of a class value against the point-charge
// limit 1/r.
//
// For a displacement d (grid units, sorted |dx| >= |dy| >= |dz|, r = |d|):
//   r <= r_cut (6)          exact (staged contraction, FP64)
//   r_cut < r <= r_mlp      1/r + s(r) * MLP(features(d))
//   r > r_mlp               1/r
// s(r) = exp(c0 + c1 r + c2 r^2) is the envelope of the residual's magnitude
// (a fit of log max |residual| per radial shell), so the network's target
// z = residual / s(r) is O(1) over the whole range.  Features: d / 16, r / 16,
// d / r.  Network: 7 -> 64 -> 64 -> 64 -> 64 -> 1, tanh on the hidden layers,
// FP32 parameters, FP32 training (full-batch Adam, cosine learning-rate
// decay, loss weighted by (s(r) / max s)^2 so that the absolute residual error
// is what the fit minimises) and FP32 inference.
//
// Evaluation of a class list: a seeded audit sample of the far classes (a
// fraction of every radial shell, at least a few classes per shell) is also
// computed exactly; every shell whose audit error exceeds the tolerance is
// computed exactly in full.  Near and audited classes always carry exact
// values.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <random>
#include <tuple>
#include <vector>

#include "gli_internal.cuh"

namespace gli {

constexpr int MLP_IN = 7, MLP_W = 64, MLP_HIDDEN = 4;
// flat parameter layout: for each layer l: W_l (out x in, row-major), then b_l
__host__ __device__ constexpr int mlp_layer_in(int l) { return l == 0 ? MLP_IN : MLP_W; }
__host__ __device__ constexpr int mlp_layer_out(int l) { return l == MLP_HIDDEN ? 1 : MLP_W; }
// closed form (no recursion: kernels keep a statically sized stack)
__host__ __device__ constexpr int mlp_offset(int l) {
    return l == 0 ? 0
                  : (MLP_W * MLP_IN + MLP_W) + (l <= MLP_HIDDEN ? l - 1 : MLP_HIDDEN - 1) * (MLP_W * MLP_W + MLP_W) +
                        (l > MLP_HIDDEN ? MLP_W + 1 : 0);
}
constexpr int MLP_PARAMS = mlp_offset(MLP_HIDDEN + 1);
constexpr int MLP_ACT = MLP_HIDDEN * MLP_W;  // stored activations per sample
static_assert(MLP_PARAMS == 7 * 64 + 64 + 3 * (64 * 64 + 64) + 64 + 1, "parameter count");
static_assert(mlp_offset(1) == 512 && mlp_offset(4) == 12992, "layer offsets");

__host__ __device__ inline void mlp_features(double a, double b, double c, float f[MLP_IN]) {
    const double r = sqrt(a * a + b * b + c * c);
    f[0] = (float)(a / 16.0);
    f[1] = (float)(b / 16.0);
    f[2] = (float)(c / 16.0);
    f[3] = (float)(r / 16.0);
    f[4] = (float)(r > 0 ? a / r : 0.0);
    f[5] = (float)(r > 0 ? b / r : 0.0);
    f[6] = (float)(r > 0 ? c / r : 0.0);
}

// forward pass of one sample; h[l * 64 + o] = tanh activations of the hidden layers
__device__ inline float mlp_forward_one(const float* __restrict__ P, const float* x, float* h) {
    const float* in = x;
    for (int l = 0; l < MLP_HIDDEN; ++l) {
        const int nin = mlp_layer_in(l);
        const float* W = P + mlp_offset(l);
        const float* b = W + MLP_W * nin;
        float* out = h + l * MLP_W;
        for (int o = 0; o < MLP_W; ++o) {
            float acc = b[o];
            for (int i = 0; i < nin; ++i) acc = fmaf(W[o * nin + i], in[i], acc);
            out[o] = tanhf(acc);
        }
        in = out;
    }
    const float* W = P + mlp_offset(MLP_HIDDEN);
    float y = W[MLP_W];
    for (int i = 0; i < MLP_W; ++i) y = fmaf(W[i], in[i], y);
    return y;
}

__global__ void k_mlp_forward(const float* __restrict__ P, const float* __restrict__ X, int n, float* __restrict__ H,
                              float* __restrict__ Y) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float h[MLP_ACT];
    Y[s] = mlp_forward_one(P, X + (i64)s * MLP_IN, h);
    for (int k = 0; k < MLP_ACT; ++k) H[(i64)s * MLP_ACT + k] = h[k];
}

// deltas (d loss / d pre-activation) of every layer of one sample:
// D[s][l * 64 + o] for the hidden layers, D[s][MLP_ACT] for the output;
// loss = sum_s w_s (y_s - t_s)^2 / sum_s w_s
__global__ void k_mlp_backward(const float* __restrict__ P, const float* __restrict__ H, const float* __restrict__ Y,
                               const float* __restrict__ T, const float* __restrict__ Wt, float inv_wsum, int n,
                               float* __restrict__ D) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float* h = H + (i64)s * MLP_ACT;
    float* d = D + (i64)s * (MLP_ACT + 1);
    const float dy = 2.0f * Wt[s] * inv_wsum * (Y[s] - T[s]);
    d[MLP_ACT] = dy;
    // last hidden layer: W_out (1 x 64)
    const float* Wo = P + mlp_offset(MLP_HIDDEN);
    float g[MLP_W];
    for (int i = 0; i < MLP_W; ++i) {
        const float a = h[(MLP_HIDDEN - 1) * MLP_W + i];
        g[i] = Wo[i] * dy * (1.0f - a * a);
        d[(MLP_HIDDEN - 1) * MLP_W + i] = g[i];
    }
    for (int l = MLP_HIDDEN - 1; l >= 1; --l) {
        const float* W = P + mlp_offset(l);  // 64 x 64: maps layer l-1 activations to layer l
        float gn[MLP_W];
        for (int i = 0; i < MLP_W; ++i) {
            float acc = 0;
            for (int o = 0; o < MLP_W; ++o) acc = fmaf(W[o * MLP_W + i], g[o], acc);
            const float a = h[(l - 1) * MLP_W + i];
            gn[i] = acc * (1.0f - a * a);
        }
        for (int i = 0; i < MLP_W; ++i) {
            g[i] = gn[i];
            d[(l - 1) * MLP_W + i] = gn[i];
        }
    }
}

// gradient of every parameter: sum over samples of delta_out * input_in
// (thread per parameter; the layer input is X for layer 0, else the previous
// layer's activations)
__global__ void k_mlp_grads(const float* __restrict__ X, const float* __restrict__ H, const float* __restrict__ D,
                            int n, float* __restrict__ G) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= MLP_PARAMS) return;
    int l = 0;
    while (l < MLP_HIDDEN && p >= mlp_offset(l + 1)) ++l;
    const int q = p - mlp_offset(l);
    const int nin = l == 0 ? MLP_IN : MLP_W, nout = l == MLP_HIDDEN ? 1 : MLP_W;
    const bool bias = q >= nout * nin;
    const int o = bias ? q - nout * nin : q / nin, i = bias ? 0 : q % nin;
    const int dcol = l == MLP_HIDDEN ? MLP_ACT : l * MLP_W + o;
    float acc = 0;
    for (int s = 0; s < n; ++s) {
        const float dv = D[(i64)s * (MLP_ACT + 1) + dcol];
        float in = 1.0f;
        if (!bias) in = l == 0 ? X[(i64)s * MLP_IN + i] : H[(i64)s * MLP_ACT + (l - 1) * MLP_W + i];
        acc = fmaf(dv, in, acc);
    }
    G[p] = acc;
}

// Adam with cosine learning-rate decay over `total` steps; step counter in device memory
__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M, float* __restrict__ V,
                       const int* __restrict__ step, int total, float lr0) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= MLP_PARAMS) return;
    const int t = *step + 1;
    const float lr = lr0 * 0.5f * (1.0f + cospif((float)t / (float)total));
    const float b1 = 0.9f, b2 = 0.999f;
    const float m = b1 * M[p] + (1 - b1) * G[p];
    const float v = b2 * V[p] + (1 - b2) * G[p] * G[p];
    M[p] = m;
    V[p] = v;
    const float mh = m / (1.0f - powf(b1, (float)t)), vh = v / (1.0f - powf(b2, (float)t));
    P[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

__global__ void k_step_inc(int* step) { *step += 1; }

// sorted |displacement| of ERIDA classes (index i N + j of the grid)
__global__ void k_erida_disp(GridDesc g, const int64_t* __restrict__ idx, i64 m, int* __restrict__ disp) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    const i64 N = g.num[0] * g.num[1] * g.num[2];
    i64 a = idx[n] / N, b = idx[n] % N;
    int p[2][3];
    for (int k = 0; k < 2; ++k) {
        i64 l = k ? b : a;
        p[k][2] = (int)(l % g.num[2]);
        l /= g.num[2];
        p[k][1] = (int)(l % g.num[1]);
        p[k][0] = (int)(l / g.num[1]);
    }
    int d[3];
    for (int ax = 0; ax < 3; ++ax) d[ax] = abs(p[0][ax] - p[1][ax]);
    if (d[0] < d[1]) { int t = d[0]; d[0] = d[1]; d[1] = t; }
    if (d[1] < d[2]) { int t = d[1]; d[1] = d[2]; d[2] = t; }
    if (d[0] < d[1]) { int t = d[0]; d[0] = d[1]; d[1] = t; }
    disp[3 * n] = d[0];
    disp[3 * n + 1] = d[1];
    disp[3 * n + 2] = d[2];
}

// slot of a sorted displacement a >= b >= c in a dense (R+1)^3 table
__host__ __device__ inline int disp_slot(int a, int b, int c, int R) { return (a * (R + 1) + b) * (R + 1) + c; }

// predicted values of classes: 1/r + s(r) MLP (r_cut < r <= r_mlp) or 1/r (r > r_mlp);
// classes with r <= r_cut get NaN (they are evaluated exactly).  shell[n]:
// floor(r) beyond r_cut, -1 within it.
__global__ void k_surrogate_values(const float* __restrict__ P, const int* __restrict__ disp, i64 m, double c0,
                                   double c1, double c2, double r_cut, double r_mlp, const uint8_t* __restrict__ known,
                                   int R, double* __restrict__ out, int* __restrict__ shell) {
    const i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m) return;
    const int ia = disp[3 * n], ib = disp[3 * n + 1], ic = disp[3 * n + 2];
    const double a = ia, b = ib, c = ic;
    const double r = sqrt(a * a + b * b + c * c);
    // within r_cut, or a displacement the network is known to miss: exact
    if (r <= r_cut || (known && r <= r_mlp && ia <= R && known[disp_slot(ia, ib, ic, R)])) {
        out[n] = nan("");
        shell[n] = -1;
        return;
    }
    shell[n] = (int)floor(r);
    double v = 1.0 / r;
    if (r <= r_mlp) {
        float f[MLP_IN], h[MLP_ACT];
        mlp_features(a, b, c, f);
        const float z = mlp_forward_one(P, f, h);
        v += exp(c0 + c1 * r + c2 * r * r) * (double)z;
    }
    out[n] = v;
}

// ---------------------------------------------------------------------------
// host side
struct Surrogate {
    std::vector<float> params;
    double env[3] = {0, 0, 0};
    double r_cut = 6, r_mlp = 12;
    // training report
    i64 samples = 0, holdout = 0;
    double loss = 0, max_dz_train = 0, max_dz_holdout = 0, max_res_err_train = 0, max_res_err_holdout = 0;
    // |prediction - exact| of every displacement of the network's range (the
    // training and the hold-out ones: their exact values are known), indexed
    // by disp_slot(a, b, c) with a >= b >= c, dense over a <= R = ceil(r_mlp)
    int R = 0;
    std::vector<float> fit_err;
};

// One optimisation run: full-batch Adam over `steps` steps, each step a CUDA
// graph of five kernels, replayed.  Params in/out (host).
static void mlp_train_device(std::vector<float>& params, const std::vector<float>& X, const std::vector<float>& T,
                             const std::vector<float>& Wt, int steps, float lr0, cudaStream_t s) {
    const int n = (int)T.size();
    if (n <= 0) fail(GLI_ERR_ARGUMENT, "no training samples");
    double wsum = 0;
    for (float w : Wt) wsum += w;
    DevBuf<float> dP(MLP_PARAMS, s), dG(MLP_PARAMS, s), dM(MLP_PARAMS, s), dV(MLP_PARAMS, s);
    DevBuf<float> dX((i64)n * MLP_IN, s), dT(n, s), dW(n, s), dH((i64)n * MLP_ACT, s), dY(n, s),
        dD((i64)n * (MLP_ACT + 1), s);
    DevBuf<int> step(1, s);
    GLI_CUDA(cudaMemcpyAsync(dP.p, params.data(), MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(dX.p, X.data(), X.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(dT.p, T.data(), T.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(dW.p, Wt.data(), Wt.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    dM.zero();
    dV.zero();
    step.zero();
    const unsigned sb = (unsigned)((n + 127) / 128), pb = (unsigned)((MLP_PARAMS + 255) / 256);
    auto one_step = [&]() {
        k_mlp_forward<<<sb, 128, 0, s>>>(dP.p, dX.p, n, dH.p, dY.p);
        k_mlp_backward<<<sb, 128, 0, s>>>(dP.p, dH.p, dY.p, dT.p, dW.p, (float)(1.0 / wsum), n, dD.p);
        k_mlp_grads<<<pb, 256, 0, s>>>(dX.p, dH.p, dD.p, n, dG.p);
        k_adam<<<pb, 256, 0, s>>>(dP.p, dG.p, dM.p, dV.p, step.p, steps, lr0);
        k_step_inc<<<1, 1, 0, s>>>(step.p);
    };
    // one step as a graph, replayed
    GLI_CUDA(cudaStreamSynchronize(s));  // the host vectors above were copied
    GLI_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    one_step();
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    GLI_CUDA(cudaGetLastError());
    GLI_CUDA(ce);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    GLI_CUDA(ie);
    cudaError_t le = cudaSuccess;
    for (int t = 0; t < steps && le == cudaSuccess; ++t) le = cudaGraphLaunch(exec, s);
    const cudaError_t se = le == cudaSuccess ? cudaStreamSynchronize(s) : le;
    cudaGraphExecDestroy(exec);
    GLI_CUDA(se);
    add_launches(5LL * steps);
    GLI_CUDA(cudaMemcpyAsync(params.data(), dP.p, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
}

static void mlp_predict_device(const std::vector<float>& params, const std::vector<float>& X, std::vector<float>& Y,
                               cudaStream_t s) {
    const int n = (int)(X.size() / MLP_IN);
    Y.assign(n, 0.f);
    if (n == 0) return;
    DevBuf<float> dP(MLP_PARAMS, s), dX((i64)n * MLP_IN, s), dH((i64)n * MLP_ACT, s), dY(n, s);
    GLI_CUDA(cudaMemcpyAsync(dP.p, params.data(), MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(dX.p, X.data(), X.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    k_mlp_forward<<<(n + 127) / 128, 128, 0, s>>>(dP.p, dX.p, n, dH.p, dY.p);
    GLI_CHECK_LAUNCH();
    GLI_CUDA(cudaMemcpyAsync(Y.data(), dY.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
}

// exact ERIDA values of host class indices on a grid (FP64 form)
static std::vector<double> exact_erida(const double* coeffs, i64 nb, const GridDesc& g, const std::vector<int64_t>& idx,
                                       double tol, cudaStream_t s) {
    std::vector<double> out(idx.size());
    if (idx.empty()) return out;
    DevBuf<int64_t> di((i64)idx.size(), s);
    DevBuf<double> dv((i64)idx.size(), s);
    GLI_CUDA(cudaMemcpyAsync(di.p, idx.data(), idx.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    sparse_values_device(0, coeffs, nb, g, di.p, (i64)idx.size(), tol, FORM_FP64, dv.p, s, nullptr);
    GLI_CUDA(cudaMemcpyAsync(out.data(), dv.p, idx.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    return out;
}

static GridDesc cube(int L) {
    GridDesc g;
    for (int a = 0; a < 3; ++a) {
        g.istart[a] = -(L / 2);
        g.num[a] = L;
    }
    return g;
}

// class index on a centred cube of edge L for displacement (a, b, c): points (0,0,0) and (a,b,c)
static int64_t erida_index(int L, int a, int b, int c) {
    const i64 e = L / 2, N = (i64)L * L * L;
    auto lin = [&](i64 x, i64 y, i64 z) { return ((x + e) * L + (y + e)) * L + (z + e); };
    const i64 i = lin(0, 0, 0), j = lin(a, b, c);
    return i * N + j;
}

Surrogate* surrogate_train(const double* coeffs, i64 nb, double tol, double r_mlp, int steps, double lr,
                           double holdout_fraction, uint64_t seed, cudaStream_t s) {
    if (!(r_mlp > 6.0) || r_mlp > 64) fail(GLI_ERR_ARGUMENT, "r_mlp must lie in (6, 64]");
    if (steps < 1 || steps > 10000000) fail(GLI_ERR_ARGUMENT, "steps must lie in 1 .. 1e7");
    if (!(holdout_fraction >= 0 && holdout_fraction < 0.9)) fail(GLI_ERR_ARGUMENT, "holdout fraction in [0, 0.9)");
    auto sur = new Surrogate;
    std::unique_ptr<Surrogate> guard(sur);
    sur->r_mlp = r_mlp;
    // Training classes: displacements with r_cut < r <= r_mlp, evaluated exactly
    // on the odd centred cubes 25^3, 33^3, 49^3 and 65^3 (the smallest cube
    // that holds a displacement evaluates it; every displacement of the range
    // occurs on the 25^3 cube and gives the same value on every larger one)
    const int edges[4] = {25, 33, 49, 65};
    std::map<std::tuple<int, int, int>, int> seen;
    std::vector<std::tuple<int, int, int>> disp;
    std::vector<int> cube_of;
    const int R = (int)ceil(r_mlp);
    for (int a = 0; a <= R; ++a)
        for (int b = 0; b <= a; ++b)
            for (int c = 0; c <= b; ++c) {
                const double r = sqrt((double)a * a + (double)b * b + (double)c * c);
                if (!(r > sur->r_cut && r <= r_mlp)) continue;
                int e = -1;
                for (int k = 0; k < 4; ++k)
                    if (a <= edges[k] / 2) {
                        e = k;
                        break;
                    }
                if (e < 0) continue;
                disp.push_back({a, b, c});
                cube_of.push_back(e);
            }
    const i64 n = (i64)disp.size();
    std::vector<double> val(n);
    for (int k = 0; k < 4; ++k) {
        std::vector<int64_t> idx;
        std::vector<i64> pos;
        for (i64 q = 0; q < n; ++q)
            if (cube_of[q] == k) {
                idx.push_back(erida_index(edges[k], std::get<0>(disp[q]), std::get<1>(disp[q]), std::get<2>(disp[q])));
                pos.push_back(q);
            }
        const std::vector<double> v = exact_erida(coeffs, nb, cube(edges[k]), idx, tol, s);
        for (size_t q = 0; q < pos.size(); ++q) val[pos[q]] = v[q];
    }
    // residuals, envelope of log max |res| per shell (least-squares quadratic)
    std::vector<double> r(n), res(n);
    std::map<int, double> shell_max;
    for (i64 q = 0; q < n; ++q) {
        const double a = std::get<0>(disp[q]), b = std::get<1>(disp[q]), c = std::get<2>(disp[q]);
        r[q] = sqrt(a * a + b * b + c * c);
        res[q] = val[q] - 1.0 / r[q];
        const int sh = (int)floor(r[q]);
        shell_max[sh] = std::max(shell_max[sh], fabs(res[q]));
    }
    {
        double S[5] = {0, 0, 0, 0, 0}, Y[3] = {0, 0, 0};
        int cnt = 0;
        for (auto& kv : shell_max) {
            if (!(kv.second > 0)) continue;
            const double x = kv.first + 0.5, y = log(kv.second);
            double p = 1;
            for (int k = 0; k < 5; ++k) {
                S[k] += p;
                if (k < 3) Y[k] += p * y;
                p *= x;
            }
            ++cnt;
        }
        if (cnt < 3) fail(GLI_ERR_INTERNAL, "too few shells for the residual envelope");
        // normal equations of the quadratic fit, solved by Cramer's rule
        const double A[3][3] = {{S[0], S[1], S[2]}, {S[1], S[2], S[3]}, {S[2], S[3], S[4]}};
        auto det3 = [](const double M[3][3]) {
            return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                   M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        };
        const double d0 = det3(A);
        for (int k = 0; k < 3; ++k) {
            double B[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) B[i][j] = j == k ? Y[i] : A[i][j];
            sur->env[k] = det3(B) / d0;
        }
    }
    // samples: features, targets z = res / s(r), weights (s / max s)^2
    std::vector<float> X(n * MLP_IN), T(n), W(n);
    double smax = 0;
    std::vector<double> env(n);
    for (i64 q = 0; q < n; ++q) {
        env[q] = exp(sur->env[0] + sur->env[1] * r[q] + sur->env[2] * r[q] * r[q]);
        smax = std::max(smax, env[q]);
    }
    for (i64 q = 0; q < n; ++q) {
        mlp_features(std::get<0>(disp[q]), std::get<1>(disp[q]), std::get<2>(disp[q]), &X[q * MLP_IN]);
        T[q] = (float)(res[q] / env[q]);
        W[q] = (float)std::max(1e-4, (env[q] / smax) * (env[q] / smax));
    }
    // seeded hold-out split
    std::mt19937_64 rng(seed);
    std::vector<i64> perm(n);
    for (i64 q = 0; q < n; ++q) perm[q] = q;
    std::shuffle(perm.begin(), perm.end(), rng);
    const i64 nh = (i64)(holdout_fraction * n);
    std::vector<float> Xt, Tt, Wtr, Xh;
    std::vector<i64> hold(perm.begin(), perm.begin() + nh), train(perm.begin() + nh, perm.end());
    for (i64 q : train) {
        Xt.insert(Xt.end(), &X[q * MLP_IN], &X[q * MLP_IN] + MLP_IN);
        Tt.push_back(T[q]);
        Wtr.push_back(W[q]);
    }
    for (i64 q : hold) Xh.insert(Xh.end(), &X[q * MLP_IN], &X[q * MLP_IN] + MLP_IN);
    // initial parameters: N(0, 1 / fan-in) weights, zero biases (seeded)
    sur->params.assign(MLP_PARAMS, 0.f);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (int l = 0; l <= MLP_HIDDEN; ++l) {
        const int nin = mlp_layer_in(l), nout = mlp_layer_out(l);
        for (int k = 0; k < nin * nout; ++k) sur->params[mlp_offset(l) + k] = (float)(nd(rng) / sqrt((double)nin));
    }
    mlp_train_device(sur->params, Xt, Tt, Wtr, steps, (float)lr, s);
    // report
    std::vector<float> yt, yh;
    mlp_predict_device(sur->params, Xt, yt, s);
    mlp_predict_device(sur->params, Xh, yh, s);
    double wsum = 0, loss = 0;
    for (size_t k = 0; k < train.size(); ++k) {
        const i64 q = train[k];
        const double dz = (double)yt[k] - T[q];
        loss += W[q] * dz * dz;
        wsum += W[q];
        sur->max_dz_train = std::max(sur->max_dz_train, fabs(dz));
        sur->max_res_err_train = std::max(sur->max_res_err_train, fabs((double)yt[k] * env[q] - res[q]));
    }
    for (size_t k = 0; k < hold.size(); ++k) {
        const i64 q = hold[k];
        sur->max_dz_holdout = std::max(sur->max_dz_holdout, fabs((double)yh[k] - T[q]));
        sur->max_res_err_holdout = std::max(sur->max_res_err_holdout, fabs((double)yh[k] * env[q] - res[q]));
    }
    sur->R = R;
    sur->fit_err.assign((size_t)(R + 1) * (R + 1) * (R + 1), 0.f);
    for (size_t k = 0; k < train.size(); ++k) {
        const i64 q = train[k];
        sur->fit_err[disp_slot(std::get<0>(disp[q]), std::get<1>(disp[q]), std::get<2>(disp[q]), R)] =
            (float)fabs((double)yt[k] * env[q] - res[q]);
    }
    for (size_t k = 0; k < hold.size(); ++k) {
        const i64 q = hold[k];
        sur->fit_err[disp_slot(std::get<0>(disp[q]), std::get<1>(disp[q]), std::get<2>(disp[q]), R)] =
            (float)fabs((double)yh[k] * env[q] - res[q]);
    }
    sur->loss = wsum > 0 ? loss / wsum : 0;
    sur->samples = (i64)train.size();
    sur->holdout = nh;
    return guard.release();
}

void surrogate_free(Surrogate* s) { delete s; }

// Surrogate values of an ERIDA class list with the per-shell audit.  report
// (optional, max_shells x 4 doubles): per radial shell k = floor(r): classes,
// audited, max audit error, computed exactly in full (1/0).
void surrogate_erida_values(const Surrogate& sur, const double* coeffs, i64 nb, const GridDesc& g,
                            const int64_t* h_idx, i64 m, double tol, double audit_fraction, uint64_t seed,
                            double shell_tol, double* h_out, double* report, i64 max_shells, cudaStream_t s) {
    if (m <= 0) return;
    if (!(audit_fraction >= 0 && audit_fraction <= 1)) fail(GLI_ERR_ARGUMENT, "audit fraction in [0, 1]");
    if (!(shell_tol >= 0)) fail(GLI_ERR_ARGUMENT, "shell tolerance must be non-negative");
    DevBuf<int64_t> di(m, s);
    DevBuf<int> dd(3 * m, s), dsh(m, s);
    DevBuf<double> dv(m, s);
    DevBuf<float> dP(MLP_PARAMS, s);
    GLI_CUDA(cudaMemcpyAsync(di.p, h_idx, m * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(dP.p, sur.params.data(), MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, s));
    k_erida_disp<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(g, di.p, m, dd.p);
    GLI_CHECK_LAUNCH();
    // displacements whose fit error (measured at training) exceeds shell_tol
    // are evaluated exactly: the audit samples a shell, this covers the
    // outliers it may miss
    std::vector<uint8_t> known(sur.fit_err.size());
    bool any = false;
    for (size_t k = 0; k < known.size(); ++k) {
        known[k] = sur.fit_err[k] > shell_tol ? 1 : 0;
        any = any || known[k];
    }
    DevBuf<uint8_t> dknown(any ? known.size() : 0, s);
    if (any)
        GLI_CUDA(cudaMemcpyAsync(dknown.p, known.data(), known.size(), cudaMemcpyHostToDevice, s));
    k_surrogate_values<<<(unsigned)((m + 127) / 128), 128, 0, s>>>(dP.p, dd.p, m, sur.env[0], sur.env[1], sur.env[2],
                                                                    sur.r_cut, sur.r_mlp, any ? dknown.p : nullptr,
                                                                    sur.R, dv.p, dsh.p);
    GLI_CHECK_LAUNCH();
    std::vector<int> shell(m);
    GLI_CUDA(cudaMemcpyAsync(h_out, dv.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaMemcpyAsync(shell.data(), dsh.p, m * sizeof(int), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    // classes bucketed by shell (counting sort, class order kept within a shell)
    int ns = 0;
    for (i64 n = 0; n < m; ++n) ns = std::max(ns, shell[n] + 1);
    std::vector<i64> first(ns + 1, 0);
    std::vector<i64> exact;
    for (i64 n = 0; n < m; ++n) {
        if (shell[n] < 0)
            exact.push_back(n);
        else
            ++first[shell[n] + 1];
    }
    for (int k = 0; k < ns; ++k) first[k + 1] += first[k];
    std::vector<i64> members(first[ns]);
    {
        std::vector<i64> fill(first.begin(), first.end() - 1);
        for (i64 n = 0; n < m; ++n)
            if (shell[n] >= 0) members[fill[shell[n]]++] = n;
    }
    // the audit sample of a shell: its k classes of smallest seeded hash of the
    // class index (splitmix64 finaliser), k = audit_fraction of the shell, at
    // least 4 (all of a smaller shell); audit_fraction 0: no audit (the
    // prediction alone, for measurements).  The hash makes the sample a
    // function of the seed and the class, not of the list order.
    auto mix = [](uint64_t z) {
        z += 0x9e3779b97f4a7c15ull;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    };
    std::vector<i64> nsample(ns, 0);
    std::vector<std::pair<uint64_t, i64>> keyed;
    for (int k = 0; k < ns; ++k) {
        const i64 cnt = first[k + 1] - first[k];
        if (cnt == 0 || audit_fraction <= 0) continue;
        const i64 want = std::min<i64>(cnt, std::max<i64>(4, (i64)ceil(audit_fraction * cnt)));
        keyed.clear();
        for (i64 q = first[k]; q < first[k + 1]; ++q)
            keyed.push_back({mix(seed ^ (uint64_t)h_idx[members[q]]), members[q]});
        if (want < cnt) std::nth_element(keyed.begin(), keyed.begin() + want, keyed.end());
        for (i64 q = 0; q < want; ++q) exact.push_back(keyed[q].second);
        nsample[k] = want;
    }
    std::vector<int64_t> eidx(exact.size());
    for (size_t k = 0; k < exact.size(); ++k) eidx[k] = h_idx[exact[k]];
    const std::vector<double> ev = exact_erida(coeffs, nb, g, eidx, tol, s);
    // audit error per shell (the audited classes follow the near ones in `exact`)
    std::vector<double> shell_err(ns, 0.0);
    for (size_t k = 0; k < exact.size(); ++k) {
        const i64 n = exact[k];
        if (shell[n] >= 0) shell_err[shell[n]] = std::max(shell_err[shell[n]], fabs(h_out[n] - ev[k]));
    }
    for (size_t k = 0; k < exact.size(); ++k) h_out[exact[k]] = ev[k];
    // shells whose audit exceeds the tolerance are evaluated exactly in full
    std::vector<int64_t> ridx;
    std::vector<i64> redo;
    for (int k = 0; k < ns; ++k) {
        if (nsample[k] == 0 || shell_err[k] <= shell_tol) continue;
        for (i64 q = first[k]; q < first[k + 1]; ++q) {
            redo.push_back(members[q]);
            ridx.push_back(h_idx[members[q]]);
        }
    }
    if (!redo.empty()) {
        const std::vector<double> rv = exact_erida(coeffs, nb, g, ridx, tol, s);
        for (size_t k = 0; k < redo.size(); ++k) h_out[redo[k]] = rv[k];
    }
    if (report && max_shells > 0) {
        for (i64 k = 0; k < 4 * max_shells; ++k) report[k] = 0;
        for (int k = 0; k < ns && k < max_shells; ++k) {
            const i64 cnt = first[k + 1] - first[k];
            if (cnt == 0) continue;
            double* rp = report + 4 * k;
            rp[0] = (double)cnt;
            rp[1] = (double)nsample[k];
            rp[2] = shell_err[k];
            rp[3] = nsample[k] > 0 && !(shell_err[k] <= shell_tol) ? 1.0 : 0.0;
        }
    }
}

// one forward + backward pass of the training kernels (no update): loss and
// gradient for the checks against a CPU restatement
void mlp_loss_grad(const float* params, const float* X, const float* T, const float* Wt, i64 n, float* loss,
                   float* grads, cudaStream_t s) {
    if (n <= 0) fail(GLI_ERR_ARGUMENT, "no samples");
    double wsum = 0;
    for (i64 k = 0; k < n; ++k) wsum += Wt[k];
    DevBuf<float> dP(MLP_PARAMS, s), dG(MLP_PARAMS, s), dX(n * MLP_IN, s), dT(n, s), dW(n, s), dH(n * MLP_ACT, s),
        dY(n, s), dD(n * (MLP_ACT + 1), s);
    GLI_CUDA(cudaMemcpyAsync(dP.p, params, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(dX.p, X, n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(dT.p, T, n * sizeof(float), cudaMemcpyHostToDevice, s));
    GLI_CUDA(cudaMemcpyAsync(dW.p, Wt, n * sizeof(float), cudaMemcpyHostToDevice, s));
    const unsigned sb = (unsigned)((n + 127) / 128);
    k_mlp_forward<<<sb, 128, 0, s>>>(dP.p, dX.p, (int)n, dH.p, dY.p);
    GLI_CHECK_LAUNCH();
    k_mlp_backward<<<sb, 128, 0, s>>>(dP.p, dH.p, dY.p, dT.p, dW.p, (float)(1.0 / wsum), (int)n, dD.p);
    GLI_CHECK_LAUNCH();
    k_mlp_grads<<<(MLP_PARAMS + 255) / 256, 256, 0, s>>>(dX.p, dH.p, dD.p, (int)n, dG.p);
    GLI_CHECK_LAUNCH();
    std::vector<float> y(n);
    GLI_CUDA(cudaMemcpyAsync(y.data(), dY.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaMemcpyAsync(grads, dG.p, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, s));
    GLI_CUDA(cudaStreamSynchronize(s));
    double l = 0;
    for (i64 k = 0; k < n; ++k) l += Wt[k] * ((double)y[k] - T[k]) * ((double)y[k] - T[k]);
    *loss = (float)(l / wsum);
}

int mlp_param_count() { return MLP_PARAMS; }

}  // namespace gli

// ---------------------------------------------------------------------------
// C entry points (no counterpart in the reference)
struct gli_b200_surrogate {
    gli::Surrogate* impl;
};

namespace {
template <class F>
int surrogate_guard(F&& f) {
    gli::clear_error();
    try {
        f();
    } catch (const gli::Failure&) {
        if (!getenv("GLI_B200_QUIET")) fprintf(stderr, "gausslectronitegrate_b200: %s\n", gli::last_message());
    } catch (const std::bad_alloc&) {
        gli::set_error(GLI_ERR_ALLOC, "host allocation failed");
    }
    return gli::last_error();
}
}  // namespace

extern "C" int gli_b200_surrogate_train(const struct gausslet_data* gdata, double tol, double r_mlp, int steps,
                                        double lr, double holdout_fraction, unsigned long long seed,
                                        gli_b200_surrogate** out) {
    return surrogate_guard([&] {
        if (!out) gli::fail(GLI_ERR_ARGUMENT, "out must not be NULL");
        *out = nullptr;
        if (!gdata || !gdata->coefficients || gdata->indices.num <= 0) gli::fail(GLI_ERR_ARGUMENT, "no coefficients");
        gli::Context& ctx = gli::context();
        gli::Surrogate* s = gli::surrogate_train(gdata->coefficients, gdata->indices.num, tol, r_mlp, steps, lr,
                                                 holdout_fraction, seed, ctx.stream);
        *out = new gli_b200_surrogate{s};
    });
}

extern "C" void gli_b200_surrogate_free(gli_b200_surrogate* s) {
    if (!s) return;
    gli::surrogate_free(s->impl);
    delete s;
}

// info[0..10]: training samples, hold-out samples, weighted loss, max |dz| train,
// max |dz| hold-out, max |residual error| train, max |residual error| hold-out,
// r_cut, r_mlp, parameter count, envelope c2 (c0, c1 follow in info[11], info[12])
extern "C" int gli_b200_surrogate_info(const gli_b200_surrogate* s, double info[13]) {
    return surrogate_guard([&] {
        if (!s || !info) gli::fail(GLI_ERR_ARGUMENT, "NULL argument");
        const gli::Surrogate& u = *s->impl;
        const double v[13] = {(double)u.samples, (double)u.holdout, u.loss, u.max_dz_train, u.max_dz_holdout,
                              u.max_res_err_train, u.max_res_err_holdout, u.r_cut, u.r_mlp,
                              (double)gli::mlp_param_count(), u.env[2], u.env[0], u.env[1]};
        memcpy(info, v, sizeof(v));
    });
}

extern "C" glong gli_b200_surrogate_params(const gli_b200_surrogate* s, float* params, glong n) {
    if (!s) return -1;
    const glong k = (glong)s->impl->params.size();
    if (params) memcpy(params, s->impl->params.data(), (size_t)std::min(k, n) * sizeof(float));
    return k;
}

extern "C" int gli_b200_erida_surrogate_values(const gli_b200_surrogate* s, const struct gausslet_data* gdata,
                                               const struct cartesian_grid_3d* grid, const glong* indices, glong num,
                                               double tol, double audit_fraction, unsigned long long seed,
                                               double shell_tol, double* values, double* report, glong max_shells) {
    return surrogate_guard([&] {
        if (!s || !gdata || !grid || (num > 0 && (!indices || !values))) gli::fail(GLI_ERR_ARGUMENT, "NULL argument");
        const gli::GridDesc g = gli::grid_desc(grid);
        gli::Context& ctx = gli::context();
        gli::surrogate_erida_values(*s->impl, gdata->coefficients, gdata->indices.num, g, (const int64_t*)indices, num,
                                    tol, audit_fraction, seed, shell_tol, values, report, max_shells, ctx.stream);
    });
}

extern "C" int gli_b200_mlp_loss_grad(const float* params, const float* X, const float* T, const float* W, glong n,
                                      float* loss, float* grads) {
    return surrogate_guard([&] {
        if (!params || !X || !T || !W || !loss || !grads) gli::fail(GLI_ERR_ARGUMENT, "NULL argument");
        gli::Context& ctx = gli::context();
        gli::mlp_loss_grad(params, X, T, W, n, loss, grads, ctx.stream);
    });
}

extern "C" int gli_b200_mlp_param_count(void) { return gli::mlp_param_count(); }
