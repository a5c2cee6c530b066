/* CPU reference of the surrogate's 3x3 convolutions (test infrastructure).
 *
 * Plain loops over NHWC float images with zero padding, weights
 * [Cout][9][Cin] (tap = ky*3 + kx), accumulation in double so the reference
 * is well below the tolerance of the bf16 tensor-core kernels it checks:
 *   y[n,y,x,co]  = sum_{ky,kx,ci} x[n,y+ky-1,x+kx-1,ci] w[co,ky,kx,ci] (+ b, ReLU)
 *   dx[n,y,x,ci] = sum_{ky,kx,co} dy[n,y-ky+1,x-kx+1,co] w[co,ky,kx,ci]
 *   dw[co,ky,kx,ci] = sum_{n,y,x} dy[n,y,x,co] x[n,y+ky-1,x+kx-1,ci]
 */
#include <stddef.h>

static inline size_t pix(int n, int y, int x, int H, int W) { return ((size_t)n * H + y) * W + x; }

void conv_ref_fwd(const float *x, int N, int H, int W, int Cin, const float *w, int Cout,
                  const float *bias, int relu, float *y)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int n = 0; n < N; n++)
        for (int yy = 0; yy < H; yy++)
            for (int xx = 0; xx < W; xx++)
                for (int co = 0; co < Cout; co++) {
                    double s = bias ? bias[co] : 0.0;
                    for (int t = 0; t < 9; t++) {
                        const int sy = yy + t / 3 - 1, sx = xx + t % 3 - 1;
                        if (sy < 0 || sy >= H || sx < 0 || sx >= W)
                            continue;
                        const float *xr = x + pix(n, sy, sx, H, W) * Cin;
                        const float *wr = w + ((size_t)co * 9 + t) * Cin;
                        for (int ci = 0; ci < Cin; ci++)
                            s += (double)xr[ci] * wr[ci];
                    }
                    if (relu && s < 0.0)
                        s = 0.0;
                    y[pix(n, yy, xx, H, W) * Cout + co] = (float)s;
                }
}

void conv_ref_dgrad(const float *dy, int N, int H, int W, int Cout, const float *w, int Cin,
                    float *dx)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int n = 0; n < N; n++)
        for (int yy = 0; yy < H; yy++)
            for (int xx = 0; xx < W; xx++)
                for (int ci = 0; ci < Cin; ci++) {
                    double s = 0.0;
                    for (int t = 0; t < 9; t++) {
                        const int oy = yy - (t / 3 - 1), ox = xx - (t % 3 - 1);
                        if (oy < 0 || oy >= H || ox < 0 || ox >= W)
                            continue;
                        const float *g = dy + pix(n, oy, ox, H, W) * Cout;
                        for (int co = 0; co < Cout; co++)
                            s += (double)g[co] * w[((size_t)co * 9 + t) * Cin + ci];
                    }
                    dx[pix(n, yy, xx, H, W) * Cin + ci] = (float)s;
                }
}

void conv_ref_wgrad(const float *dy, const float *x, int N, int H, int W, int Cin, int Cout,
                    float *dw)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int co = 0; co < Cout; co++)
        for (int t = 0; t < 9; t++)
            for (int ci = 0; ci < Cin; ci++) {
                double s = 0.0;
                for (int n = 0; n < N; n++)
                    for (int yy = 0; yy < H; yy++)
                        for (int xx = 0; xx < W; xx++) {
                            const int sy = yy + t / 3 - 1, sx = xx + t % 3 - 1;
                            if (sy < 0 || sy >= H || sx < 0 || sx >= W)
                                continue;
                            s += (double)dy[pix(n, yy, xx, H, W) * Cout + co] *
                                 x[pix(n, sy, sx, H, W) * Cin + ci];
                        }
                dw[((size_t)co * 9 + t) * Cin + ci] = (float)s;
            }
}
