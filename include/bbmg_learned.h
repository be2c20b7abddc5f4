/*
 * bbmg_learned.h -- kernels of the learned initial guess (3-D U-Net).
 *
 * No counterpart in the reference: NGA2 starts every pressure solve from the
 * previous pressure (or zero).  These entry points are the building blocks of
 * a small 3-D U-Net that predicts the pressure increment from the right-hand
 * side and the previous pressure; the network is orchestrated from the host
 * (nga2_b200/learned.py) and always followed by the multigrid solve, which
 * still decides convergence.
 *
 * Activations are BF16, channels-last: element (voxel v, channel c) of a view
 * lives at data[v * ld + c]; voxels are ordered (n, d, h, w) with w fastest and
 * every direction periodic.  Convolutions are 3x3x3 with periodic padding,
 * FP32 accumulation; channel counts are multiples of 16.  Weights: FP32
 * master copies w[tap][cin][cout] (tap = 9 dz + 3 dy + dx, offsets -1..1 as
 * 0..2), packed to BF16 by nn_pack_weights.  All pointers are device memory;
 * every call is asynchronous on `stream` and returns 0 or an error code
 * (BBMG_BAD_ARGS / BBMG_CUDA of bbmg_b200.h).
 */
#ifndef BBMG_LEARNED_H
#define BBMG_LEARNED_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    void *data;       /* __nv_bfloat16 */
    int n, d, h, w;   /* batch and spatial sizes */
    int c;            /* channels of the view */
    int ld;           /* elements between consecutive voxels (>= c, even) */
} nn_act;

/* y = act(conv3x3x3(x, w) + bias); act = ReLU when relu != 0.  wt is the
 * forward packing of nn_pack_weights.  Tensor cores with FP32 accumulation:
 * tcgen05.mma with a TMEM accumulator when the rows hold a multiple of 128
 * voxels (cout 16..64, 16-byte aligned views), mma.sync otherwise. */
int nn_conv3(const nn_act *x, const void *wt, const float *bias, const nn_act *y, int relu, void *stream);

/* BBMG_CUDA if a tcgen05 convolution's completion wait ran out since the last
 * call (the flag is then cleared), else 0.  Synchronises the device. */
int nn_tc_error(void);

/* dx = conv3x3x3 of dy with the mirrored, transposed weights (wd, the
 * backward packing): the gradient of the convolution input. */
int nn_conv3_dgrad(const nn_act *dy, const void *wd, const nn_act *dx, void *stream);

/* dw[tap][cin][cout] += sum_v x(v + tap) dy(v) and db[cout] += sum_v dy(v)
 * (FP32 accumulation; dw/db are accumulated into, zero them first).  On the
 * tensor cores (mma.sync, BF16 products) when cin % 16 == 0, cout % 8 == 0 and
 * the channel rows are 16-byte aligned; on the CUDA cores otherwise. */
int nn_conv3_wgrad(const nn_act *x, const nn_act *dy, float *dw, float *db, void *stream);

/* FP32 master weights [27][cin][cout] -> BF16 forward ([27][cout][cin]) and
 * backward ([27][cin][cout], taps mirrored) packings. */
int nn_pack_weights(const float *w, int cin, int cout, void *wt, void *wd, void *stream);

/* dy *= (y > 0): the ReLU derivative applied in place. */
int nn_relu_bwd(const nn_act *dy, const nn_act *y, void *stream);

/* 2x2x2 average pooling and nearest-neighbour upsampling, with gradients
 * (y is half / twice the spatial size of x).  nn_pool2_bwd overwrites dx, or
 * adds to it when accumulate != 0 (a pooled tensor that is also a skip
 * connection). */
int nn_pool2(const nn_act *x, const nn_act *y, void *stream);
int nn_pool2_bwd(const nn_act *dy, const nn_act *dx, int accumulate, void *stream);
int nn_up2(const nn_act *x, const nn_act *y, void *stream);
int nn_up2_bwd(const nn_act *dy, const nn_act *dx, void *stream);

/* Input embedding: channel i = scales[i] * fields[i] for i < nf, the other
 * channels 0, from nf (<= NN_MAX_FIELDS) FP64 fields (w fastest).  With
 * pool = 1 the fields have x's n*d*h*w values; with pool = 2 they live on the
 * grid twice as fine (n, 2d, 2h, 2w) and are averaged over 2x2x2 children.
 * fields and scales are host arrays; the fields are device memory. */
#define NN_MAX_FIELDS 4
int nn_embed(int nf, const double *const *fields, const double *scales, int pool, const nn_act *x, void *stream);

/* 1x1x1 head: out[v] = b + sum_c x(v,c) w[c] (FP32 out).  Backward: dx(v,c) =
 * dout[v] w[c] (BF16), dw[c] += sum_v dout[v] x(v,c), db += sum_v dout[v]. */
int nn_head(const nn_act *x, const float *w, const float *b, float *out, void *stream);
int nn_head_bwd(const nn_act *x, const float *w, const float *dout, const nn_act *dx, float *dw, float *db,
                void *stream);

/* Mean-squared error of pred against scale * target (FP64 field): writes
 * dloss/dpred = 2 (pred - scale*target) / nvox and accumulates sum of squares
 * into *loss (zero it first). */
int nn_mse(const float *pred, const double *target, double scale, long long nvox, float *grad, double *loss,
           void *stream);

/* Adam step on n FP32 parameters (step t >= 1). */
int nn_adam(float *w, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
            int t, void *stream);

/* out = base + scale * pred (FP64 out; base may be NULL for 0): the predicted
 * pressure.  pred is (nb, d, h, w); out is (nb, up*d, up*h, up*w).  up = 2
 * interpolates a prediction made on the grid twice as coarse trilinearly
 * between cell centres (periodic). */
int nn_apply(const double *base, const float *pred, double scale, int nb, int d, int h, int w, int up, double *out,
             void *stream);

#ifdef __cplusplus
}
#endif
#endif /* BBMG_LEARNED_H */
