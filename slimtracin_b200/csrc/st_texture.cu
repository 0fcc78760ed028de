// st_texture.cu — loadTexture (bmp2texture.c:324) on the device: an 8-bit RGB(A) image -> the
// reference's residency format, a chain of TexelQuad grids ((w+1) x (h+1) quads of 2x2 texels).
//
// The reference works in float texels: mip 0 is the image, each further mip (while both sides are
// above 4) box-filters the one before, summing TL + TR + BL + BR in that order and scaling by 0.25
// (bmp2texture.c:284-306), and only the final quads are truncated to u8 (:346-361).  The quads are
// written by a scatter loop over texels with edge replication (bmp2texture.c:181-237) whose later
// writes overwrite earlier ones on the border; the device gathers instead, one thread per quad,
// with the source texel each quadrant ends up holding:
//   left  x-1 (wrap: w-1 at x = 0;  clamp: 0)      top    y-1 (wrap: h-1 at y = 0; clamp: 0)
//   right x   (clamp: w-1 at x = w; wrap: w-1 at x = w, except the top row's TR and the bottom
//              row's BR, which keep the wrapped texel 0 — the loop's clamped writes of the last
//              column land after its wrapped ones everywhere else)
//   bottom y  (wrap: 0 at y = h;    clamp: h-1)
#include <algorithm>
#include "st_kernels.h"

namespace st {

namespace {

__global__ void unpack_kernel(const uint8_t *components, u32t n, int stride, float *texels) {
    const u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t *c = components + (size_t)i * stride;
    texels[3 * (size_t)i] = (float)c[0];
    texels[3 * (size_t)i + 1] = (float)c[1];
    texels[3 * (size_t)i + 2] = (float)c[2];
}

// Next mip: 2x2 box filter of the previous mip's float texels (bmp2texture.c:289-303).
__global__ void downsample_kernel(const float *src, u32t src_w, float *dst, u32t w, u32t h) {
    const u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const u32t x = i % w, y = i / w;
    const float *tl = src + 3 * ((size_t)(2 * y) * src_w + 2 * x);
    const float *tr = tl + 3;
    const float *bl = tl + 3 * (size_t)src_w;
    const float *br = bl + 3;
    for (int c = 0; c < 3; c++) {
        float s = tl[c];
        s += tr[c];
        s += bl[c];
        s += br[c];
        dst[3 * (size_t)i + c] = s * 0.25f;
    }
}

__global__ void quads_kernel(const float *texels, u32t w, u32t h, int wrap, TexelQuad *out) {
    const u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    const u32t qw = w + 1;
    if (i >= qw * (h + 1)) return;
    const u32t qx = i % qw, qy = i / qw;
    u32t left, top, bottom, right_tr, right_br;
    if (wrap) {
        left = qx == 0 ? w - 1 : qx - 1;
        top = qy == 0 ? h - 1 : qy - 1;
        bottom = qy == h ? 0 : qy;
        right_tr = qx == w ? (qy == 0 ? 0 : w - 1) : qx;
        right_br = qx == w ? (qy == h ? 0 : w - 1) : qx;
    } else {
        left = qx == 0 ? 0 : qx - 1;
        top = qy == 0 ? 0 : qy - 1;
        bottom = qy == h ? h - 1 : qy;
        right_tr = right_br = qx == w ? w - 1 : qx;
    }
    const float *tl = texels + 3 * ((size_t)top * w + left);
    const float *tr = texels + 3 * ((size_t)top * w + right_tr);
    const float *bl = texels + 3 * ((size_t)bottom * w + left);
    const float *br = texels + 3 * ((size_t)bottom * w + right_br);
    TexelQuad q;
    q.R.TL = (u8)tl[0]; q.G.TL = (u8)tl[1]; q.B.TL = (u8)tl[2];
    q.R.TR = (u8)tr[0]; q.G.TR = (u8)tr[1]; q.B.TR = (u8)tr[2];
    q.R.BL = (u8)bl[0]; q.G.BL = (u8)bl[1]; q.B.BL = (u8)bl[2];
    q.R.BR = (u8)br[0]; q.G.BR = (u8)br[1]; q.B.BR = (u8)br[2];
    out[i] = q;
}

}  // namespace

int texture_mip_count(u32t width, u32t height, bool mipmap) {
    int n = 1;
    if (mipmap)
        while (width > 4 && height > 4) {
            width /= 2;
            height /= 2;
            n++;
        }
    return n;
}

size_t texture_quad_count(u32t width, u32t height, bool mipmap) {
    size_t q = 0;
    const int n = texture_mip_count(width, height, mipmap);
    for (int m = 0; m < n; m++, width /= 2, height /= 2) q += (size_t)(width + 1) * (height + 1);
    return q;
}

size_t texture_scratch_bytes(u32t width, u32t height) {
    // two float texel planes (current and next mip) and the image
    return 2 * (3 * sizeof(float) * (size_t)width * height + 256) + 4 * (size_t)width * height + 256;
}

cudaError_t bake_texture(const uint8_t *dev_components, u32t width, u32t height, int bit_count, bool wrap, bool mipmap,
                         void *scratch, TexelQuad *dev_quads, cudaStream_t st) {
    const u32t T = 256;
    float *cur = static_cast<float *>(scratch);
    float *next = cur + (3 * (size_t)width * height + 63) / 64 * 64;
    const u32t n = width * height;
    unpack_kernel<<<(n + T - 1) / T, T, 0, st>>>(dev_components, n, bit_count == 32 ? 4 : 3, cur);
    const int mips = texture_mip_count(width, height, mipmap);
    u32t w = width, h = height;
    TexelQuad *out = dev_quads;
    for (int m = 0; m < mips; m++) {
        const u32t quads = (w + 1) * (h + 1);
        quads_kernel<<<(quads + T - 1) / T, T, 0, st>>>(cur, w, h, wrap ? 1 : 0, out);
        out += quads;
        if (m + 1 < mips) {
            downsample_kernel<<<((w / 2) * (h / 2) + T - 1) / T, T, 0, st>>>(cur, w, next, w / 2, h / 2);
            std::swap(cur, next);
            w /= 2;
            h /= 2;
        }
    }
    return cudaGetLastError();
}

}  // namespace st
