// Warm-start network: a periodic 3-D convolutional encoder-decoder that maps a solute's
// potential channels (3 x N) to projections of the converged log-density: the 4 m <= 1
// real-basis projections (nout = 4), or the real and imaginary parts of all np complex
// projections of the solver's angular grid (nout = 2 np).  Forward, backward and Adam run on the device with the kernels of
// k_warmnet.cuh; the host here owns the parameters, the activation buffers and the
// launch order.  There is no counterpart in the reference (it always starts from the
// bulk guess, src/module_density.f90:267-284).
//
// Network (grid n^3 with n divisible by 8; levels n, n/2, n/4, n/8):
//   e0a conv3 3->16, e0b conv3 16->16          level 0    (GELU after every conv3/down)
//   d1 down 16->32, e1 conv3 32->32            level 1
//   d2 down 32->64, e2 conv3 64->64            level 2
//   d3 down 64->128, m conv3 128->128          level 3
//   u2 up 128->64 + e2, c2 conv3 64->64        level 2    (up: linear, then the skip add)
//   u1 up 64->32 + e1, c1 conv3 32->32         level 1
//   u0 up 32->16 + e0b, c0 conv3 16->16        level 0
//   head conv1 16->nout (linear)
// 906,772 parameters at nout = 4 (weights and biases), BF16 in the kernels, FP32 master
// copy for Adam.
#include "../../include/mdft_b200.h"

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "k_warmnet.cuh"

using namespace mdft;
using namespace mdft::wn;

namespace {

enum Kind { kConv3 = 0, kDown = 1, kUp = 2, kHead = 3 };
struct TensorSpec { int c, level; };
struct LayerSpec { int kind, x, y, cin, cout, skip, gelu; };

constexpr int kNT = 16;  // tensors: 0 = input channels, 15 = output projections
constexpr int kNL = 15;  // layers
const TensorSpec kTensors[kNT] = {{3, 0},  {16, 0}, {16, 0}, {32, 1}, {32, 1}, {64, 2},  {64, 2}, {128, 3},
                                  {128, 3}, {64, 2}, {64, 2}, {32, 1}, {32, 1}, {16, 0}, {16, 0}, {4, 0}};
const LayerSpec kLayers[kNL] = {
    {kConv3, 0, 1, 3, 16, -1, 1},     {kConv3, 1, 2, 16, 16, -1, 1},   {kDown, 2, 3, 16, 32, -1, 1},
    {kConv3, 3, 4, 32, 32, -1, 1},    {kDown, 4, 5, 32, 64, -1, 1},    {kConv3, 5, 6, 64, 64, -1, 1},
    {kDown, 6, 7, 64, 128, -1, 1},    {kConv3, 7, 8, 128, 128, -1, 1}, {kUp, 8, 9, 128, 64, 6, 0},
    {kConv3, 9, 10, 64, 64, -1, 1},   {kUp, 10, 11, 64, 32, 4, 0},     {kConv3, 11, 12, 32, 32, -1, 1},
    {kUp, 12, 13, 32, 16, 2, 0},      {kConv3, 13, 14, 16, 16, -1, 1}, {kHead, 14, 15, 16, 4, -1, 0},
};

int kvol(int kind) { return kind == kConv3 ? 27 : (kind == kHead ? 1 : 8); }
long long nweights(const LayerSpec &L) { return (long long)L.cin * L.cout * kvol(L.kind); }
// the layer and tensor tables with the network's own output count in the head
LayerSpec layer_of(int nout, int l) {
    LayerSpec L = kLayers[l];
    if (L.kind == kHead) L.cout = nout;
    return L;
}
int channels_of(int nout, int t) { return t == kNT - 1 ? nout : kTensors[t].c; }

int cuda_rc(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MDFT_OK;
    cudaGetLastError();
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? MDFT_E_NOMEM : MDFT_E_CUDA;
}

constexpr int kWgradTarget = 4 * 148;  // CTAs a weight-gradient launch aims for

// voxel splits of a weight-gradient reduction: (number of splits, voxels per split)
void split_plan(int K3, int cin, int cout, long long nout, int *nsplit, long long *per) {
    const long long tiles = (long long)((cin * K3 + kBM - 1) / kBM) * ((cout + kBN - 1) / kBN);
    long long ns = (kWgradTarget + tiles - 1) / tiles;
    const long long maxs = (nout + 255) / 256;
    if (ns > maxs) ns = maxs;
    if (ns < 1) ns = 1;
    long long p = (nout + ns - 1) / ns;
    p = (p + kBK - 1) / kBK * kBK;
    *per = p;
    *nsplit = (int)((nout + p - 1) / p);
}

unsigned ew_grid(long long n) {
    long long b = (n + 255) / 256;
    return (unsigned)(b < 2048 ? (b < 1 ? 1 : b) : 2048);
}

// deterministic normal deviates: splitmix64 + Box-Muller
struct Rng {
    unsigned long long s;
    unsigned long long next() {
        unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.14159265358979323846 * u2);
    }
};

}  // namespace

struct mdft_warm_net {
    int device = 0;
    int nx = 0, ny = 0, nz = 0;
    int nout = 4;  // output channels (head width)
    cudaStream_t stream = nullptr;
    cudaStream_t own = nullptr;
    long long nparam = 0;
    long long woff[kNL], boff[kNL];
    DevBuf<float> p, g, m, v;
    DevBuf<__nv_bfloat16> pb;
    DevBuf<float> act[kNT], grad[kNT], z[kNL];
    DevBuf<float> part;
    DevBuf<double> lpart, lacc;
    long long part_cap = 0;
    bool train_ready = false;
    long long loss_count = 0;
    int step = 0;
    long long launches = 0;

    Vol vol(int level) const { return Vol{nz >> level, ny >> level, nx >> level}; }
    long long nvox(int level) const { return vol(level).n(); }
    LayerSpec layer(int l) const { return layer_of(nout, l); }
    int channels(int t) const { return channels_of(nout, t); }
};

namespace {

template <int MODE, int KS, int S>
void conv(mdft_warm_net *net, const ConvArgs &a) {
    const Vol vg = MODE == kParity ? a.vin : a.vout;
    dim3 grid((unsigned)((vg.n() + kBM - 1) / kBM), (unsigned)((a.cout + kBN - 1) / kBN), MODE == kParity ? 8u : 1u);
    k_conv_gemm<MODE, KS, S><<<grid, kThreads, 0, net->stream>>>(a);
    net->launches += 1;
}

template <int KS, int S>
void wgrad(mdft_warm_net *net, const float *dy, const float *x, int cin, int cout, Vol vin, Vol vout, float *dw, int accumulate) {
    constexpr int K3 = KS * KS * KS;
    int nsplit;
    long long per;
    split_plan(K3, cin, cout, vout.n(), &nsplit, &per);
    WgradArgs a{dy, x, net->part.p, cin, cout, vin, vout, per};
    dim3 grid((unsigned)((cin * K3 + kBM - 1) / kBM), (unsigned)((cout + kBN - 1) / kBN), (unsigned)nsplit);
    k_conv_wgrad<KS, S><<<grid, kThreads, 0, net->stream>>>(a);
    const long long n = (long long)cout * cin * K3;
    k_wgrad_reduce<<<ew_grid(n), 256, 0, net->stream>>>(net->part.p, dw, nsplit, n, accumulate);
    net->launches += 2;
}

const float *tensor_in(mdft_warm_net *net, int t, const float *in) { return t == 0 ? in : net->act[t].p; }

void forward(mdft_warm_net *net, const float *in) {
    const __nv_bfloat16 *P = net->pb.p;
    for (int l = 0; l < kNL; ++l) {
        const LayerSpec L = net->layer(l);
        const int lx = kTensors[L.x].level, ly = kTensors[L.y].level;
        const float *x = tensor_in(net, L.x, in);
        float *out = L.gelu ? net->z[l].p : net->act[L.y].p;
        const __nv_bfloat16 *W = P + net->woff[l];
        const float *b = net->p.p + net->boff[l];
        ConvArgs a{x, W, b, out, L.cin, L.cout, net->vol(lx), net->vol(ly), 0};
        switch (L.kind) {
            case kConv3: conv<kFwd, 3, 1>(net, a); break;
            case kDown: conv<kFwd, 2, 2>(net, a); break;
            case kHead: conv<kFwd, 1, 1>(net, a); break;
            case kUp:
                conv<kParity, 2, 2>(net, a);
                k_add<<<ew_grid(net->nvox(ly) * L.cout), 256, 0, net->stream>>>(out, net->act[L.skip].p, net->nvox(ly) * L.cout);
                net->launches += 1;
                break;
        }
        if (L.gelu) {
            const long long n = net->nvox(ly) * L.cout;
            k_gelu<<<ew_grid(n), 256, 0, net->stream>>>(out, net->act[L.y].p, n);
            net->launches += 1;
        }
    }
}

// loss and parameter gradients of one sample (accumulated into g when accumulate)
void backward(mdft_warm_net *net, const float *in, const float *target, const float *mask, int accumulate) {
    cudaStream_t st = net->stream;
    for (int t = 1; t < kNT - 1; ++t) cudaMemsetAsync(net->grad[t].p, 0, net->grad[t].bytes(), st);
    const long long nv0 = net->nvox(0);
    const int nblk = 296;
    k_mse<<<nblk, 256, 0, st>>>(net->act[kNT - 1].p, target, mask, net->grad[kNT - 1].p, net->lpart.p, net->nout, nv0,
                                (float)(1.0 / ((double)net->nout * (double)nv0)));
    k_sum_into<<<1, 256, 0, st>>>(net->lpart.p, nblk, net->lacc.p);
    net->launches += 2;
    float *G = net->g.p;
    for (int l = kNL - 1; l >= 0; --l) {
        const LayerSpec L = net->layer(l);
        const int lx = kTensors[L.x].level, ly = kTensors[L.y].level;
        const Vol vx = net->vol(lx), vy = net->vol(ly);
        float *gy = net->grad[L.y].p;
        const long long ny = vy.n() * L.cout;
        if (L.gelu) {
            k_gelu_bwd<<<ew_grid(ny), 256, 0, st>>>(net->z[l].p, gy, ny);
            net->launches += 1;
        }
        k_bias_grad<<<L.cout, 256, 0, st>>>(gy, G + net->boff[l], vy.n(), accumulate);
        net->launches += 1;
        const float *x = tensor_in(net, L.x, in);
        const __nv_bfloat16 *W = net->pb.p + net->woff[l];
        float *dW = G + net->woff[l];
        float *gx = L.x > 0 ? net->grad[L.x].p : nullptr;
        switch (L.kind) {
            case kConv3:
                wgrad<3, 1>(net, gy, x, L.cin, L.cout, vx, vy, dW, accumulate);
                if (gx) conv<kBwdData, 3, 1>(net, ConvArgs{gy, W, nullptr, gx, L.cout, L.cin, vy, vx, 1});
                break;
            case kHead:
                wgrad<1, 1>(net, gy, x, L.cin, L.cout, vx, vy, dW, accumulate);
                if (gx) conv<kBwdData, 1, 1>(net, ConvArgs{gy, W, nullptr, gx, L.cout, L.cin, vy, vx, 1});
                break;
            case kDown:
                wgrad<2, 2>(net, gy, x, L.cin, L.cout, vx, vy, dW, accumulate);
                if (gx) conv<kParity, 2, 2>(net, ConvArgs{gy, W, nullptr, gx, L.cout, L.cin, vy, vx, 1});
                break;
            case kUp:
                k_add<<<ew_grid(ny), 256, 0, st>>>(net->grad[L.skip].p, gy, ny);
                net->launches += 1;
                // dW[cc][cf][a] = sum_o X[cc][o] dF[cf][2o + a]: the coarse input plays the
                // gradient, the fine gradient plays the input of a stride-2 convolution
                wgrad<2, 2>(net, x, gy, L.cout, L.cin, vy, vx, dW, accumulate);
                if (gx) conv<kFwd, 2, 2>(net, ConvArgs{gy, W, nullptr, gx, L.cout, L.cin, vy, vx, 1});
                break;
        }
    }
}

int ensure_train(mdft_warm_net *net) {
    if (net->train_ready) return MDFT_OK;
    int rc;
    const size_t n = (size_t)net->nparam;
    if ((rc = cuda_rc(net->g.alloc(n), "gradients"))) return rc;
    if ((rc = cuda_rc(net->m.alloc(n), "Adam m"))) return rc;
    if ((rc = cuda_rc(net->v.alloc(n), "Adam v"))) return rc;
    cudaMemsetAsync(net->m.p, 0, n * 4, net->stream);
    cudaMemsetAsync(net->v.p, 0, n * 4, net->stream);
    for (int t = 1; t < kNT; ++t) {
        const size_t c = (size_t)net->channels(t) * net->nvox(kTensors[t].level);
        if ((rc = cuda_rc(net->grad[t].alloc(c), "activation gradients"))) return rc;
    }
    long long cap = 1;
    for (int l = 0; l < kNL; ++l) {
        const LayerSpec L = net->layer(l);
        int ns;
        long long per;
        const int K3 = kvol(L.kind);
        if (L.kind == kUp) {
            split_plan(K3, L.cout, L.cin, net->nvox(kTensors[L.x].level), &ns, &per);
        } else {
            split_plan(K3, L.cin, L.cout, net->nvox(kTensors[L.y].level), &ns, &per);
        }
        const long long need = (long long)ns * L.cin * L.cout * K3;
        if (need > cap) cap = need;
    }
    if ((rc = cuda_rc(net->part.alloc((size_t)cap), "weight-gradient partials"))) return rc;
    net->part_cap = cap;
    if ((rc = cuda_rc(net->lpart.alloc(296), "loss partials"))) return rc;
    net->train_ready = true;
    net->step = 0;
    return cuda_rc(cudaGetLastError(), "training buffers");
}

int check_net(const mdft_warm_net *net) {
    if (!net) { set_error("null network"); return MDFT_E_ARG; }
    return MDFT_OK;
}

}  // namespace

extern "C" {

int mdft_warm_net_create(int nx, int ny, int nz, int device, mdft_warm_net **out) {
    return mdft_warm_net_create_n(nx, ny, nz, 4, device, out);
}

int mdft_warm_net_create_n(int nx, int ny, int nz, int nout, int device, mdft_warm_net **out) {
    if (!out) { set_error("null argument"); return MDFT_E_ARG; }
    *out = nullptr;
    if (nout < 1 || nout > 256) { set_error("warm-start network outputs %d: must be in [1, 256]", nout); return MDFT_E_ARG; }
    if (nx < 8 || ny < 8 || nz < 8 || nx % 8 || ny % 8 || nz % 8) {
        set_error("warm-start network grid %dx%dx%d: every dimension must be a multiple of 8", nx, ny, nz);
        return MDFT_E_ARG;
    }
    int rc = cuda_rc(cudaSetDevice(device), "cudaSetDevice");
    if (rc) return rc;
    mdft_warm_net *net = new mdft_warm_net;
    net->device = device;
    net->nx = nx; net->ny = ny; net->nz = nz;
    net->nout = nout;
    long long off = 0;
    for (int l = 0; l < kNL; ++l) {
        net->woff[l] = off;
        off += nweights(net->layer(l));
        net->boff[l] = off;
        off += net->layer(l).cout;
    }
    net->nparam = off;
    auto fail = [&](int r) { delete net; return r; };
    if ((rc = cuda_rc(cudaStreamCreateWithFlags(&net->own, cudaStreamNonBlocking), "stream"))) return fail(rc);
    net->stream = net->own;
    if ((rc = cuda_rc(net->p.alloc((size_t)off), "parameters"))) return fail(rc);
    if ((rc = cuda_rc(net->pb.alloc((size_t)off), "BF16 parameters"))) return fail(rc);
    cudaMemsetAsync(net->p.p, 0, (size_t)off * 4, net->stream);
    cudaMemsetAsync(net->pb.p, 0, (size_t)off * 2, net->stream);
    for (int t = 1; t < kNT; ++t) {
        const size_t c = (size_t)net->channels(t) * net->nvox(kTensors[t].level);
        if ((rc = cuda_rc(net->act[t].alloc(c), "activations"))) return fail(rc);
    }
    for (int l = 0; l < kNL; ++l)
        if (kLayers[l].gelu) {
            const size_t c = (size_t)net->layer(l).cout * net->nvox(kTensors[kLayers[l].y].level);
            if ((rc = cuda_rc(net->z[l].alloc(c), "pre-activations"))) return fail(rc);
        }
    if ((rc = cuda_rc(net->lacc.alloc(1), "loss"))) return fail(rc);
    cudaMemsetAsync(net->lacc.p, 0, 8, net->stream);
    if ((rc = cuda_rc(cudaStreamSynchronize(net->stream), "network create"))) return fail(rc);
    *out = net;
    return MDFT_OK;
}

int mdft_warm_net_destroy(mdft_warm_net *net) {
    if (!net) return MDFT_OK;
    cudaSetDevice(net->device);
    if (net->stream) cudaStreamSynchronize(net->stream);
    cudaStream_t own = net->own;
    delete net;
    if (own) cudaStreamDestroy(own);
    return MDFT_OK;
}

int mdft_warm_net_num_params(const mdft_warm_net *net, long long *n) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!n) { set_error("null argument"); return MDFT_E_ARG; }
    *n = net->nparam;
    return MDFT_OK;
}

int mdft_warm_net_set_stream(mdft_warm_net *net, void *stream) {
    int rc = check_net(net);
    if (rc) return rc;
    net->stream = stream ? (cudaStream_t)stream : net->own;
    return MDFT_OK;
}

int mdft_warm_net_set_params(mdft_warm_net *net, const float *params, long long n) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!params || n != net->nparam) {
        set_error("parameter vector of %lld values, the network has %lld", n, net->nparam);
        return MDFT_E_ARG;
    }
    for (long long i = 0; i < n; ++i)
        if (!std::isfinite(params[i])) { set_error("non-finite parameter %lld", i); return MDFT_E_NUMERIC; }
    if ((rc = cuda_rc(cudaMemcpyAsync(net->p.p, params, (size_t)n * 4, cudaMemcpyHostToDevice, net->stream), "parameters upload")))
        return rc;
    k_to_bf16<<<ew_grid(n), 256, 0, net->stream>>>(net->p.p, net->pb.p, n);
    net->launches += 1;
    if (net->train_ready) {
        cudaMemsetAsync(net->m.p, 0, (size_t)n * 4, net->stream);
        cudaMemsetAsync(net->v.p, 0, (size_t)n * 4, net->stream);
        net->step = 0;
    }
    return cuda_rc(cudaStreamSynchronize(net->stream), "parameters upload");
}

int mdft_warm_net_get_params(const mdft_warm_net *net, float *params, long long n) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!params || n != net->nparam) {
        set_error("parameter vector of %lld values, the network has %lld", n, net->nparam);
        return MDFT_E_ARG;
    }
    if ((rc = cuda_rc(cudaMemcpyAsync(params, net->p.p, (size_t)n * 4, cudaMemcpyDeviceToHost, net->stream), "parameters download")))
        return rc;
    return cuda_rc(cudaStreamSynchronize(net->stream), "parameters download");
}

int mdft_warm_net_init(mdft_warm_net *net, unsigned long long seed) {
    int rc = check_net(net);
    if (rc) return rc;
    std::vector<float> h((size_t)net->nparam, 0.f);
    Rng r{seed};
    for (int l = 0; l < kNL; ++l) {
        const LayerSpec L = net->layer(l);
        // He-normal: fan-in = the inputs one output sums (the coarse channels for up-sampling)
        const double fan = L.kind == kUp ? (double)L.cin : (double)L.cin * kvol(L.kind);
        const double sd = (L.kind == kHead ? 0.1 : 1.0) * std::sqrt((L.kind == kHead ? 1.0 : 2.0) / fan);
        for (long long i = 0; i < nweights(L); ++i) h[(size_t)(net->woff[l] + i)] = (float)(sd * r.normal());
    }
    return mdft_warm_net_set_params(net, h.data(), net->nparam);
}

int mdft_warm_net_forward(mdft_warm_net *net, const float *d_in, float *d_out) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!d_in) { set_error("null input"); return MDFT_E_ARG; }
    forward(net, d_in);
    if (d_out) {
        const size_t bytes = net->act[kNT - 1].bytes();
        if ((rc = cuda_rc(cudaMemcpyAsync(d_out, net->act[kNT - 1].p, bytes, cudaMemcpyDeviceToDevice, net->stream), "output copy")))
            return rc;
    }
    return cuda_rc(cudaGetLastError(), "network forward");
}

int mdft_warm_net_output(mdft_warm_net *net, const float **d_out) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!d_out) { set_error("null argument"); return MDFT_E_ARG; }
    *d_out = net->act[kNT - 1].p;
    return MDFT_OK;
}

int mdft_warm_net_gradients(mdft_warm_net *net, const float *d_in, const float *d_target, const float *d_mask, float *grad,
                            double *loss) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!d_in || !d_target || !grad) { set_error("null argument"); return MDFT_E_ARG; }
    if ((rc = ensure_train(net))) return rc;
    cudaMemsetAsync(net->lacc.p, 0, 8, net->stream);
    forward(net, d_in);
    backward(net, d_in, d_target, d_mask, 0);
    if ((rc = cuda_rc(cudaGetLastError(), "network backward"))) return rc;
    cudaMemcpyAsync(grad, net->g.p, (size_t)net->nparam * 4, cudaMemcpyDeviceToHost, net->stream);
    double l = 0.0;
    cudaMemcpyAsync(&l, net->lacc.p, 8, cudaMemcpyDeviceToHost, net->stream);
    cudaMemsetAsync(net->lacc.p, 0, 8, net->stream);
    if ((rc = cuda_rc(cudaStreamSynchronize(net->stream), "network gradients"))) return rc;
    net->loss_count = 0;
    if (loss) *loss = l;
    return MDFT_OK;
}

int mdft_warm_net_train_step(mdft_warm_net *net, const float *const *d_in, const float *const *d_target,
                             const float *const *d_mask, int nbatch, float lr) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!d_in || !d_target || nbatch <= 0 || !(lr > 0.f)) { set_error("invalid training batch"); return MDFT_E_ARG; }
    for (int i = 0; i < nbatch; ++i)
        if (!d_in[i] || !d_target[i]) { set_error("null sample %d", i); return MDFT_E_ARG; }
    if ((rc = ensure_train(net))) return rc;
    for (int i = 0; i < nbatch; ++i) {
        forward(net, d_in[i]);
        backward(net, d_in[i], d_target[i], d_mask ? d_mask[i] : nullptr, i > 0);
    }
    net->loss_count += nbatch;
    net->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, net->step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, net->step)));
    k_adam<<<ew_grid(net->nparam), 256, 0, net->stream>>>(net->p.p, net->g.p, net->m.p, net->v.p, net->pb.p, net->nparam, lr,
                                                          b1, b2, 1e-8f, c1, c2, 1.0f / (float)nbatch);
    net->launches += 1;
    return cuda_rc(cudaGetLastError(), "training step");
}

int mdft_warm_net_take_loss(mdft_warm_net *net, double *mean_loss) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!mean_loss) { set_error("null argument"); return MDFT_E_ARG; }
    double l = 0.0;
    cudaMemcpyAsync(&l, net->lacc.p, 8, cudaMemcpyDeviceToHost, net->stream);
    cudaMemsetAsync(net->lacc.p, 0, 8, net->stream);
    if ((rc = cuda_rc(cudaStreamSynchronize(net->stream), "loss read"))) return rc;
    *mean_loss = net->loss_count > 0 ? l / (double)net->loss_count : l;
    net->loss_count = 0;
    return MDFT_OK;
}

int mdft_warm_net_launch_count(const mdft_warm_net *net, long long *count) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!count) { set_error("null argument"); return MDFT_E_ARG; }
    *count = net->launches;
    return MDFT_OK;
}

int mdft_warm_net_num_outputs(const mdft_warm_net *net, int *nout) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!nout) { set_error("null argument"); return MDFT_E_ARG; }
    *nout = net->nout;
    return MDFT_OK;
}

int mdft_warm_net_grid(const mdft_warm_net *net, int *nxyz) {
    int rc = check_net(net);
    if (rc) return rc;
    if (!nxyz) { set_error("null argument"); return MDFT_E_ARG; }
    nxyz[0] = net->nx; nxyz[1] = net->ny; nxyz[2] = net->nz;
    return MDFT_OK;
}

}  // extern "C"
