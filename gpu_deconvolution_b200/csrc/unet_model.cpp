// The warm-start network: a 4-level 2-D U-Net (3x3 convolutions, ReLU,
// base 32 channels doubling per level, 2x2 average pooling, nearest
// upsampling, additive skip connections) that maps the registered view
// planes of one z-plane, plus their mean, to an estimate of the plane.
// BF16 weights and activations, FP32 accumulation on the tensor cores
// (unet_gemm.cu), FP32 master weights trained with Adam on an L1 loss.
//
// Inputs are scaled per plane by s = 1 + mean of the views' samples; the
// network works in those units and the estimate is multiplied back by s.
//
// Layer list (index: name, input -> output channels; C_l = base << l):
//   0, 1   encoder level 0: patches(9 (V + 1), padded to 64) -> C0, C0 -> C0
//   2..7   encoder levels 1..3: pool, C_(l-1) -> C_l, C_l -> C_l
//   8..13  decoder levels 2, 1, 0: upsample, C_(l+1) -> C_l (+ skip from the
//          encoder, then ReLU), C_l -> C_l
//   then a 1 x 1 output layer C0 -> 1.
// Parameters are stored per layer as weights [cout][taps][cin] then bias.
#include "fmvd_b200.h"
#include "fmvd_internal.h"
#include "unet.h"
#include "unet_layers.h"

#include <math.h>
#include <random>
#include <string.h>
#include <vector>

namespace fmvd {
namespace unet {

using bf16 = __nv_bfloat16;

struct Layer {
    int cin, cout, taps;
    size_t w_off, b_off;  // into the parameter vector
    bf16 *wf, *wt;        // bf16 forward and data-gradient weights
};

struct Net {
    int H, W, V, maxN, base;
    std::vector<Layer> L;
    size_t out_w, out_b, nparams;
    float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
    bf16 *wbuf = nullptr;
    int step = 0;
    // activations and their gradients (maxN planes)
    bf16 *col = nullptr;
    bf16 *Ea[4], *Eb[4], *P[3], *U[3], *Da[3], *Db[3];
    bf16 *gEa[4], *gEb[4], *gP[3], *gU[3], *gDa[3], *gDb[3];
    float *scale = nullptr, *gy = nullptr, *loss = nullptr;
    float *clip = nullptr;  // adaptive gradient clipping state (3 floats)
    int *status = nullptr;
    std::vector<void *> allocs;
};

namespace {

int C_(const Net &n, int l) { return n.base << l; }
int H_(const Net &n, int l) { return n.H >> l; }
int W_(const Net &n, int l) { return n.W >> l; }
int enc_a(int l) { return 2 * l; }
int enc_b(int l) { return 2 * l + 1; }
int dec_a(int l) { return 8 + 2 * (2 - l); }
int dec_b(int l) { return 9 + 2 * (2 - l); }

template <typename T>
bool dalloc(Net &n, T **p, size_t count)
{
    void *q = nullptr;
    if (!FMVD_CHECK(cudaMalloc(&q, count * sizeof(T) + 16)))
        return false;
    n.allocs.push_back(q);
    *p = (T *)q;
    return true;
}

void release(Net *n)
{
    for (void *p : n->allocs)
        cudaFree(p);
    delete n;
}

bool conv(const Net &n, const Layer &l, const bf16 *in, int level, int N, bf16 *out, const bf16 *add, cudaStream_t s)
{
    ConvDesc c{};
    c.in = in;
    c.weight = l.wf;
    c.N = N;
    c.H = H_(n, level);
    c.W = W_(n, level);
    c.cin = l.cin;
    c.cout = l.cout;
    c.taps = l.taps;
    c.out = out;
    c.bias = n.params + l.b_off;
    c.add = add;
    c.relu = 1;
    c.status = n.status;
    return conv_forward(c, s);
}

// data gradient of layer l: g_in = conv(g_out, flipped weights), masked by
// the layer input's activation (null: no ReLU in front of the layer)
bool dgrad(const Net &n, const Layer &l, const bf16 *g_out, int level, int N, bf16 *g_in, const bf16 *mask,
           cudaStream_t s)
{
    ConvDesc c{};
    c.in = g_out;
    c.weight = l.wt;
    c.N = N;
    c.H = H_(n, level);
    c.W = W_(n, level);
    c.cin = l.cout;
    c.cout = l.cin;
    c.taps = l.taps;
    c.out = g_in;
    c.mask = mask;
    c.status = n.status;
    return conv_forward(c, s);
}

bool wgrad(const Net &n, const Layer &l, const bf16 *g_out, const bf16 *in, int level, int N, cudaStream_t s)
{
    WgradDesc c{};
    c.grad = g_out;
    c.in = in;
    c.N = N;
    c.H = H_(n, level);
    c.W = W_(n, level);
    c.cin = l.cin;
    c.cout = l.cout;
    c.taps = l.taps;
    c.dw = n.grads + l.w_off;
    c.status = n.status;
    return conv_wgrad(c, s) && bias_grad(g_out, (size_t)N * c.H * c.W, l.cout, n.grads + l.b_off, s);
}

bool refresh_weights(Net &n, cudaStream_t s)
{
    bool ok = true;
    for (size_t i = 0; i < n.L.size() && ok; i++) {
        const Layer &l = n.L[i];
        ok = weight_copies(n.params + l.w_off, l.cout, l.taps, l.cin, l.wf, i == 0 ? nullptr : l.wt, s);
    }
    return ok;
}

bool forward(Net &n, const unsigned short *views, size_t vs, int N, float *estimate, const float *target,
             cudaStream_t s)
{
    const int H = n.H, W = n.W;
    bool ok = plane_scale(views, vs, n.V, N, H * W, n.scale, s) &&
              input_patches(views, vs, n.V, N, H, W, n.scale, n.col, s) &&
              conv(n, n.L[enc_a(0)], n.col, 0, N, n.Ea[0], nullptr, s) &&
              conv(n, n.L[enc_b(0)], n.Ea[0], 0, N, n.Eb[0], nullptr, s);
    for (int l = 1; l < 4 && ok; l++)
        ok = avgpool(n.Eb[l - 1], n.P[l - 1], N, H_(n, l - 1), W_(n, l - 1), C_(n, l - 1), s) &&
             conv(n, n.L[enc_a(l)], n.P[l - 1], l, N, n.Ea[l], nullptr, s) &&
             conv(n, n.L[enc_b(l)], n.Ea[l], l, N, n.Eb[l], nullptr, s);
    for (int l = 2; l >= 0 && ok; l--) {
        const bf16 *src = l == 2 ? n.Eb[3] : n.Db[l + 1];
        ok = upsample(src, n.U[l], N, H_(n, l + 1), W_(n, l + 1), C_(n, l + 1), s) &&
             conv(n, n.L[dec_a(l)], n.U[l], l, N, n.Da[l], n.Eb[l], s) &&
             conv(n, n.L[dec_b(l)], n.Da[l], l, N, n.Db[l], nullptr, s);
    }
    if (ok && target)
        ok = FMVD_CHECK(cudaMemsetAsync(n.loss, 0, sizeof(float), s));
    return ok && output_layer(n.Db[0], n.params + n.out_w, n.params + n.out_b, n.base, N, H * W, n.scale, estimate,
                              target, n.gy, n.loss, s);
}

bool backward(Net &n, int N, cudaStream_t s)
{
    const int H = n.H, W = n.W;
    bool ok = output_grad(n.Db[0], n.params + n.out_w, n.base, (size_t)N * H * W, n.gy, n.gDb[0],
                          n.grads + n.out_w, n.grads + n.out_b, s);
    // decoder, from the output level up
    for (int l = 0; l < 3 && ok; l++) {
        const Layer &lb = n.L[dec_b(l)], &la = n.L[dec_a(l)];
        ok = wgrad(n, lb, n.gDb[l], n.Da[l], l, N, s) && dgrad(n, lb, n.gDb[l], l, N, n.gDa[l], n.Da[l], s) &&
             wgrad(n, la, n.gDa[l], n.U[l], l, N, s) && dgrad(n, la, n.gDa[l], l, N, n.gU[l], nullptr, s);
        if (ok) {
            const bf16 *src = l == 2 ? n.Eb[3] : n.Db[l + 1];
            bf16 *g_src = l == 2 ? n.gEb[3] : n.gDb[l + 1];
            ok = upsample_grad(n.gU[l], src, g_src, N, H_(n, l + 1), W_(n, l + 1), C_(n, l + 1), s);
        }
    }
    // encoder, from the bottom level down
    for (int l = 3; l >= 0 && ok; l--) {
        if (l < 3)  // pooled output gradient plus the decoder's skip gradient
            ok = pool_grad(n.gP[l], n.gDa[l], n.Eb[l], n.gEb[l], N, H_(n, l), W_(n, l), C_(n, l), s);
        const Layer &lb = n.L[enc_b(l)], &la = n.L[enc_a(l)];
        const bf16 *in_a = l == 0 ? n.col : n.P[l - 1];
        ok = ok && wgrad(n, lb, n.gEb[l], n.Ea[l], l, N, s) && dgrad(n, lb, n.gEb[l], l, N, n.gEa[l], n.Ea[l], s) &&
             wgrad(n, la, n.gEa[l], in_a, l, N, s);
        if (ok && l > 0)
            ok = dgrad(n, la, n.gEa[l], l, N, n.gP[l - 1], nullptr, s);
    }
    return ok;
}

bool check_status(Net &n)
{
    int st = 0;
    if (!FMVD_CHECK(cudaMemcpy(&st, n.status, sizeof(int), cudaMemcpyDeviceToHost)))
        return false;
    if (st) {
        cudaMemset(n.status, 0, sizeof(int));
        report_error("fmvd: a tensor-core convolution wait timed out");
        return false;
    }
    return true;
}

} // namespace

Net *create(int H, int W, int V, int maxN, unsigned seed)
{
    const int base = 32;
    // the coarsest level (H / 8 x W / 8) must tile into 128-pixel blocks
    const bool w_ok = W == 128 || W == 256 || W == 512 || (W % 1024 == 0 && W > 0);
    if (H < 128 || H % 64 || !w_ok || V < 1 || 9 * (V + 1) > kInputChannels || maxN < 1 || base > kMaxOutChannels) {
        report_error("fmvd: unsupported warm-start network geometry (height a multiple of 64, at least 128; width "
                     "128, 256, 512 or a multiple of 1024; 1 to 6 views)");
        return nullptr;
    }
    Net *n = new Net();
    n->H = H;
    n->W = W;
    n->V = V;
    n->maxN = maxN;
    n->base = base;
    size_t off = 0;
    auto add = [&](int cin, int cout, int taps) {
        Layer l{cin, cout, taps, off, 0, nullptr, nullptr};
        off += (size_t)cout * taps * cin;
        l.b_off = off;
        off += cout;
        n->L.push_back(l);
    };
    add(kInputChannels, base, 1);
    add(base, base, 9);
    for (int l = 1; l < 4; l++) {
        add(base << (l - 1), base << l, 9);
        add(base << l, base << l, 9);
    }
    for (int l = 2; l >= 0; l--) {
        add(base << (l + 1), base << l, 9);
        add(base << l, base << l, 9);
    }
    n->out_w = off;
    off += base;
    n->out_b = off;
    off += 1;
    n->nparams = off;

    // He-normal weights (fan-in of the real inputs), zero biases; the output
    // layer starts near the identity of the views' mean level
    std::vector<float> h(off, 0.f);
    std::mt19937 rng(seed);
    for (size_t i = 0; i < n->L.size(); i++) {
        const Layer &l = n->L[i];
        const int fan_in = i == 0 ? 9 * (V + 1) : l.taps * l.cin;
        std::normal_distribution<float> nd(0.f, sqrtf(2.f / (float)fan_in));
        for (int co = 0; co < l.cout; co++)
            for (int t = 0; t < l.taps; t++)
                for (int ci = 0; ci < l.cin; ci++)
                    h[l.w_off + ((size_t)co * l.taps + t) * l.cin + ci] =
                        (i == 0 && ci >= 9 * (V + 1)) ? 0.f : nd(rng);
    }
    std::normal_distribution<float> nd_out(0.f, 0.01f);
    for (int c = 0; c < base; c++)
        h[n->out_w + c] = nd_out(rng);
    h[n->out_b] = 1.f;

    size_t wtotal = 0;
    for (const Layer &l : n->L)
        wtotal += 2 * (size_t)l.cout * l.taps * l.cin;
    bool ok = dalloc(*n, &n->params, off) && dalloc(*n, &n->grads, off) && dalloc(*n, &n->m, off) &&
              dalloc(*n, &n->v, off) && dalloc(*n, &n->wbuf, wtotal) && dalloc(*n, &n->scale, (size_t)maxN * (kScaleParts + 1)) &&
              dalloc(*n, &n->gy, (size_t)maxN * H * W) && dalloc(*n, &n->loss, 1) && dalloc(*n, &n->status, 1) &&
              dalloc(*n, &n->clip, 3);
    if (ok) {
        bf16 *w = n->wbuf;
        for (Layer &l : n->L) {
            const size_t c = (size_t)l.cout * l.taps * l.cin;
            l.wf = w;
            l.wt = w + c;
            w += 2 * c;
        }
    }
    const size_t N = maxN;
    ok = ok && dalloc(*n, &n->col, N * H * W * kInputChannels);
    for (int l = 0; l < 4 && ok; l++) {
        const size_t px = N * (H >> l) * (W >> l);
        const size_t c = (size_t)base << l;
        ok = dalloc(*n, &n->Ea[l], px * c) && dalloc(*n, &n->Eb[l], px * c) && dalloc(*n, &n->gEa[l], px * c) &&
             dalloc(*n, &n->gEb[l], px * c);
        if (ok && l < 3) {
            const size_t pxp = N * (H >> (l + 1)) * (W >> (l + 1));
            ok = dalloc(*n, &n->P[l], pxp * c) && dalloc(*n, &n->gP[l], pxp * c) &&
                 dalloc(*n, &n->U[l], px * 2 * c) && dalloc(*n, &n->gU[l], px * 2 * c) &&
                 dalloc(*n, &n->Da[l], px * c) && dalloc(*n, &n->Db[l], px * c) && dalloc(*n, &n->gDa[l], px * c) &&
                 dalloc(*n, &n->gDb[l], px * c);
        }
    }
    ok = ok && FMVD_CHECK(cudaMemcpy(n->params, h.data(), off * sizeof(float), cudaMemcpyHostToDevice)) &&
         FMVD_CHECK(cudaMemset(n->m, 0, off * sizeof(float))) && FMVD_CHECK(cudaMemset(n->v, 0, off * sizeof(float))) &&
         FMVD_CHECK(cudaMemset(n->grads, 0, off * sizeof(float))) && FMVD_CHECK(cudaMemset(n->status, 0, sizeof(int))) &&
         FMVD_CHECK(cudaMemset(n->clip, 0, 3 * sizeof(float))) &&
         refresh_weights(*n, 0) && FMVD_CHECK(cudaDeviceSynchronize());
    if (!ok) {
        release(n);
        return nullptr;
    }
    return n;
}

void destroy(Net *n)
{
    if (!n)
        return;
    cudaDeviceSynchronize();
    release(n);
}

bool infer(Net *n, const unsigned short *views, size_t vs, int nplanes, float *estimate, cudaStream_t s)
{
    bool ok = true;
    for (int z0 = 0; z0 < nplanes && ok; z0 += n->maxN) {
        const int N = nplanes - z0 < n->maxN ? nplanes - z0 : n->maxN;
        ok = forward(*n, views + (size_t)z0 * n->H * n->W, vs, N, estimate + (size_t)z0 * n->H * n->W, nullptr, s);
    }
    return ok;
}

bool train_step(Net *n, const unsigned short *views, size_t vs, int N, const float *target, float lr, float *h_loss,
                cudaStream_t s)
{
    if (N > n->maxN) {
        report_error("fmvd: training batch larger than the network's maximum batch");
        return false;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    bool ok = FMVD_CHECK(cudaMemsetAsync(n->grads, 0, n->nparams * sizeof(float), s)) &&
              forward(*n, views, vs, N, nullptr, target, s) && backward(*n, N, s);
    if (ok && lr > 0.f) {
        n->step++;
        const float lr_t = lr * sqrtf(1.f - powf(b2, (float)n->step)) / (1.f - powf(b1, (float)n->step));
        // adaptive clipping keeps a rare outsized gradient (a loss spike
        // that otherwise set training back by several epochs) from
        // scattering the weights
        ok = adam(n->params, n->grads, n->m, n->v, n->nparams, lr_t, b1, b2, eps, s, n->clip, 2.f) &&
             refresh_weights(*n, s);
    }
    if (ok && h_loss)
        ok = FMVD_CHECK(cudaMemcpyAsync(h_loss, n->loss, sizeof(float), cudaMemcpyDeviceToHost, s)) &&
             FMVD_CHECK(cudaStreamSynchronize(s));
    return ok && check_status(*n);
}

} // namespace unet
} // namespace fmvd

struct fmvd_b200_unet {
    fmvd::unet::Net *net;
};

extern "C" {

fmvd_b200_unet *fmvd_b200_unet_create(int H, int W, int views, int max_batch, unsigned seed)
{
    fmvd::unet::Net *n = fmvd::unet::create(H, W, views, max_batch, seed);
    return n ? new fmvd_b200_unet{n} : nullptr;
}

void fmvd_b200_unet_destroy(fmvd_b200_unet *u)
{
    if (!u)
        return;
    fmvd::unet::destroy(u->net);
    delete u;
}

size_t fmvd_b200_unet_param_count(const fmvd_b200_unet *u) { return u ? u->net->nparams : 0; }

int fmvd_b200_unet_get_params(const fmvd_b200_unet *u, float *h_params)
{
    if (!u || !h_params)
        return 1;
    return FMVD_CHECK(cudaMemcpy(h_params, u->net->params, u->net->nparams * sizeof(float), cudaMemcpyDeviceToHost))
               ? 0
               : 1;
}

int fmvd_b200_unet_set_params(fmvd_b200_unet *u, const float *h_params)
{
    if (!u || !h_params)
        return 1;
    fmvd::unet::Net *n = u->net;
    return FMVD_CHECK(cudaMemcpy(n->params, h_params, n->nparams * sizeof(float), cudaMemcpyHostToDevice)) &&
                   fmvd::unet::refresh_weights(*n, 0) && FMVD_CHECK(cudaDeviceSynchronize())
               ? 0
               : 1;
}

int fmvd_b200_unet_get_grads(const fmvd_b200_unet *u, float *h_grads)
{
    if (!u || !h_grads)
        return 1;
    return FMVD_CHECK(cudaMemcpy(h_grads, u->net->grads, u->net->nparams * sizeof(float), cudaMemcpyDeviceToHost))
               ? 0
               : 1;
}

int fmvd_b200_unet_forward(fmvd_b200_unet *u, const void *d_views, size_t view_stride, int nplanes,
                           float *d_estimate, void *stream)
{
    if (!u || !d_views || !d_estimate || nplanes < 0) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_unet_forward");
        return 1;
    }
    return fmvd::unet::infer(u->net, (const unsigned short *)d_views, view_stride, nplanes, d_estimate,
                             (cudaStream_t)stream)
               ? 0
               : 1;
}

int fmvd_b200_unet_check(fmvd_b200_unet *u)
{
    if (!u)
        return 1;
    return fmvd::unet::check_status(*u->net) ? 0 : 1;
}

int fmvd_b200_unet_train_step(fmvd_b200_unet *u, const void *d_views, size_t view_stride, int nplanes,
                              const float *d_target, float lr, float *h_loss, void *stream)
{
    if (!u || !d_views || !d_target || nplanes < 1) {
        fmvd::report_error("fmvd: invalid arguments to fmvd_b200_unet_train_step");
        return 1;
    }
    return fmvd::unet::train_step(u->net, (const unsigned short *)d_views, view_stride, nplanes, d_target, lr, h_loss,
                                  (cudaStream_t)stream)
               ? 0
               : 1;
}

} // extern "C"
