// pt_strict.cu - wavefront path-tracing kernels in WL_MATH_STRICT mode. Built with -fmad=false
// -prec-div=true -prec-sqrt=true -ftz=false and the project's own sin/cos/log, so every path
// is bit-identical to the CPU oracle for the same inputs. Also holds the film, tone-map and
// random-stream kernels, which are exact in both modes.
#define WL_STRICT_MATH 1
#define WL_NS strict
#include "pt_kernels.cuh"

namespace wl {
namespace strict {

// Film update in path order (PathTracing.cu:145-154): per pixel, the samples of this wave in
// increasing frame; FP32 storage, double arithmetic. A path whose radiance is not finite adds 0
// (the reference would keep the NaN in its running mean). The FP64 film sums the same values.
__global__ void k_film(WaveParams wp, Queues q, Film f) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t lim = wp.count < wp.npix ? wp.count : wp.npix;
    if (j >= lim) return;
    uint64_t g0 = wp.base + j;
    uint32_t pixel = (uint32_t)(g0 % wp.npix);
    float acc[3];
    double sum[3] = {0.0, 0.0, 0.0};
    if (f.rgb)
        for (int c = 0; c < 3; c++) acc[c] = f.rgb[3 * (size_t)pixel + c];
    for (uint64_t g = g0; g < wp.base + wp.count; g += wp.npix) {
        uint32_t slot = (uint32_t)(g - wp.base);
        uint32_t frame = wp.first_frame + (uint32_t)(g / wp.npix);
        float4 r = q.st_rad[slot];
        float rc[3] = {r.x, r.y, r.z};
        if (!(isfinite(rc[0]) && isfinite(rc[1]) && isfinite(rc[2]))) rc[0] = rc[1] = rc[2] = 0.f;
        for (int c = 0; c < 3; c++) {
            if (frame == 0) {
                acc[c] = rc[c];
            } else {
                double w0 = (double)((float)frame / ((float)frame + 1.0f));
                double w1 = (double)(1.0f / ((float)frame + 1.0f));
                acc[c] = (float)((double)acc[c] * w0 + (double)rc[c] * w1);
            }
            sum[c] += (double)rc[c];
        }
    }
    if (f.rgb)
        for (int c = 0; c < 3; c++) f.rgb[3 * (size_t)pixel + c] = acc[c];
    if (f.sum64)
        for (int c = 0; c < 3; c++) f.sum64[3 * (size_t)pixel + c] += sum[c];
}

// colorBuffer = u8vec4(vec4(AceApprox(clamp(radiance, 0, 1e30)), 1) * 255) (PathTracing.cu:157-158)
__global__ void k_tonemap(Film f) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= f.W * f.H) return;
    v3 r = ld3(f.rgb + 3 * (size_t)p);
    auto gc = [](float x) {  // glm::clamp(x, 0, 1e30)
        float t = (x < 0.0f) ? 0.0f : x;
        return (1e30f < t) ? 1e30f : t;
    };
    v3 o = ace(v3(gc(r.x), gc(r.y), gc(r.z)));
    uchar4 c;
    c.x = (uint8_t)(o.x * 255.0f);
    c.y = (uint8_t)(o.y * 255.0f);
    c.z = (uint8_t)(o.z * 255.0f);
    c.w = 255;
    reinterpret_cast<uchar4 *>(f.ldr)[p] = c;
}

__global__ void k_debug_rng(uint32_t mode, uint64_t seed, const uint32_t *pixels, uint32_t npix,
                            uint32_t frame, uint32_t count, float *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    Rng r = make_rng(mode, seed, pixels[i], frame);
    for (uint32_t k = 0; k < count; k++) out[(size_t)i * count + k] = r.next();
}

void launch_film(const WaveParams &wp, const Queues &q, const Film &f, cudaStream_t s) {
    uint32_t lim = wp.count < wp.npix ? wp.count : wp.npix;
    k_film<<<(lim + 255) / 256, 256, 0, s>>>(wp, q, f);
}
void launch_tonemap(const Film &f, cudaStream_t s) {
    uint32_t n = f.W * f.H;
    k_tonemap<<<(n + 255) / 256, 256, 0, s>>>(f);
}
void launch_debug_rng(uint32_t rng, uint64_t seed, const uint32_t *pixels, uint32_t npix,
                      uint32_t frame, uint32_t count, float *out, cudaStream_t s) {
    k_debug_rng<<<(npix + 127) / 128, 128, 0, s>>>(rng, seed, pixels, npix, frame, count, out);
}

}  // namespace strict
}  // namespace wl
