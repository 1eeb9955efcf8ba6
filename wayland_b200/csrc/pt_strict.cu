// pt_strict.cu - wavefront path-tracing and bidirectional kernels in WL_MATH_STRICT mode. Built with -fmad=false
// -prec-div=true -prec-sqrt=true -ftz=false and the project's own sin/cos/log, so every path
// is bit-identical to the CPU oracle for the same inputs. Also holds the film, tone-map and
// random-stream kernels, which are exact in both modes.
#define WL_STRICT_MATH 1
#define WL_NS strict
#include <cub/device/device_scan.cuh>

#include "pt_kernels.cuh"
#include "bdpt_kernels.cuh"

namespace wl {
namespace strict {

// Film update in path order (PathTracing.cu:145-154): per pixel, the samples of this wave in
// increasing frame; FP32 storage, double arithmetic. A path whose radiance is not finite adds 0
// (the reference would keep the NaN in its running mean). The FP64 film sums the same values.
__global__ void k_film(WaveParams wp, Queues q, Film f) {
    wave_dyn(wp);
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

// Connections of a bidirectional wave: n_eye * n_light per slot, numbered by an exclusive scan in
// slot order (conn_first), and each connection tagged with its slot.
__global__ void k_bd_count(uint32_t count, BdptWave bw) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) bw.conn_count[i] = bw.n_eye[i] * bw.n_light[i];
}
__global__ void k_bd_expand(uint32_t count, BdptWave bw) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        uint32_t f = bw.conn_first[i], n = bw.conn_count[i];
        for (uint32_t k = 0; k < n; k++) bw.conn_slot[f + k] = i;
        if (i == count - 1) {
            bw.counters[0] = f + n;
            bw.counters[2] = 0;
        }
    }
}

size_t bdpt_scan_bytes(uint32_t cap) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (uint32_t *)nullptr, (uint32_t *)nullptr, (int)cap);
    return bytes;
}

void launch_bdpt_connections(const WaveParams &wp, const BdptWave &bw, cudaStream_t s) {
    uint32_t blocks = (wp.count + 255) / 256;
    k_bd_count<<<blocks ? blocks : 1, 256, 0, s>>>(wp.count, bw);
    size_t bytes = bw.scan_bytes;
    cub::DeviceScan::ExclusiveSum(bw.scan_tmp, bytes, bw.conn_count, bw.conn_first, (int)wp.count, s);
    k_bd_expand<<<blocks ? blocks : 1, 256, 0, s>>>(wp.count, bw);
}

// Film update of a bidirectional wave (BDPT.cu:534-556): per pixel, the samples of this wave in
// increasing frame; the sample is (0 + eye-path emission) + (0 + connection values in the
// reference's order), the running mean is FP32 arithmetic with FP32 weights. A sample that is
// not finite adds 0 (the reference would keep the NaN). The FP64 film sums the same values.
__global__ void k_bd_film(WaveParams wp, uint32_t nlight, Queues q, BdptWave bw, Film f) {
    wave_dyn(wp);
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
        v3 r = v3(0.f) + f4xyz(q.st_rad[slot]);
        uint32_t n = bw.conn_count[slot];
        if (n > 0 && nlight > 0) {
            v3 conn(0.f);
            uint32_t first = bw.conn_first[slot];
            for (uint32_t t = 0; t < n; t++) conn = conn + f4xyz(bw.conn_val[first + t]);
            r = r + conn;
        }
        float rc[3] = {r.x, r.y, r.z};
        if (!(isfinite(rc[0]) && isfinite(rc[1]) && isfinite(rc[2]))) rc[0] = rc[1] = rc[2] = 0.f;
        for (int c = 0; c < 3; c++) {
            if (frame == 0) {
                acc[c] = rc[c];
            } else {
                float w0 = (float)frame / ((float)frame + 1.0f);
                float w1 = 1.0f / ((float)frame + 1.0f);
                acc[c] = acc[c] * w0 + rc[c] * w1;
            }
            sum[c] += (double)rc[c];
        }
    }
    if (f.rgb)
        for (int c = 0; c < 3; c++) f.rgb[3 * (size_t)pixel + c] = acc[c];
    if (f.sum64)
        for (int c = 0; c < 3; c++) f.sum64[3 * (size_t)pixel + c] += sum[c];
}

void launch_bdpt_film(const WaveParams &wp, const DevScene &sc, const Queues &q, const BdptWave &bw,
                      const Film &f, cudaStream_t s) {
    uint32_t lim = wp.count < wp.npix ? wp.count : wp.npix;
    k_bd_film<<<(lim + 255) / 256, 256, 0, s>>>(wp, sc.nLight, q, bw, f);
}

// Film update of a batch wave: per job, per pixel, the job's samples of this wave in increasing
// frame (the same arithmetic as k_film). Thread i leads pixel g % npix of its job when g is
// among the first npix samples of the job in this wave.
__global__ void k_film_batch(BatchView bv, Queues q, uint32_t count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const BatchJob &J = bv.jobs[bv.slot_job[i]];
    const WaveParams &wp = J.wp;
    const uint64_t G = bv.wave_base + i;
    const uint64_t seg_lo = (bv.wave_base > J.off ? bv.wave_base : J.off) - J.off;
    const uint64_t wave_end = bv.wave_base + count, job_end = J.off + J.n;
    const uint64_t seg_hi = (wave_end < job_end ? wave_end : job_end) - J.off;
    const uint64_t g0 = G - J.off;
    if (g0 >= seg_lo + wp.npix) return;
    const Film &f = J.film;
    uint32_t pixel = (uint32_t)(g0 % wp.npix);
    float acc[3];
    double sum[3] = {0.0, 0.0, 0.0};
    if (f.rgb)
        for (int c = 0; c < 3; c++) acc[c] = f.rgb[3 * (size_t)pixel + c];
    for (uint64_t g = g0; g < seg_hi; g += wp.npix) {
        uint32_t slot = (uint32_t)(g + J.off - bv.wave_base);
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

void launch_film_batch(const BatchView &bv, const Queues &q, uint32_t count, cudaStream_t s) {
    k_film_batch<<<(count + 255) / 256, 256, 0, s>>>(bv, q, count);
}

// Emitter CDF of WL_LIGHTS_POWER, in FP64 and in a fixed summation order (the oracle sums in the
// same order, so both select the same triangle for every random number): emissive triangle i
// (light order, each light's triangles in order) has weight area_i * luminance(L) (Rec. 709
// weights); chunks of 256 are summed sequentially, then the chunk sums sequentially, then
// cdf_i = (chunk-local sum + chunk offset) / total, so the last entry is exactly 1.
constexpr uint32_t EMIT_CHUNK = 256;
__device__ __forceinline__ double emit_lum(const DevLight &l) {
    return 0.2126 * (double)l.L[0] + 0.7152 * (double)l.L[1] + 0.0722 * (double)l.L[2];
}
__global__ void k_emit_chunks(const float *V, const uint4 *tri, const uint32_t *emit_tri,
                              const uint32_t *emit_light, uint32_t n, const DevLight *lights,
                              double *cdf, double *chunk) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if ((uint64_t)c * EMIT_CHUNK >= n) return;
    double acc = 0.0;
    uint32_t end = (c + 1) * EMIT_CHUNK < n ? (c + 1) * EMIT_CHUNK : n;
    for (uint32_t i = c * EMIT_CHUNK; i < end; i++) {
        uint4 t = tri[emit_tri[i]];
        double ax = V[3 * (size_t)t.x], ay = V[3 * (size_t)t.x + 1], az = V[3 * (size_t)t.x + 2];
        double e1x = V[3 * (size_t)t.y] - ax, e1y = V[3 * (size_t)t.y + 1] - ay, e1z = V[3 * (size_t)t.y + 2] - az;
        double e2x = V[3 * (size_t)t.z] - ax, e2y = V[3 * (size_t)t.z + 1] - ay, e2z = V[3 * (size_t)t.z + 2] - az;
        double cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
        double area = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
        acc = acc + area * emit_lum(lights[emit_light[i]]);
        cdf[i] = acc;
    }
    chunk[c] = acc;
}
__global__ void k_emit_offsets(uint32_t chunks, double *chunk, DevLight *lights, uint32_t nLight) {
    double off = 0.0;
    for (uint32_t c = 0; c < chunks; c++) {
        double v = chunk[c];
        chunk[c] = off;
        off = off + v;
    }
    chunk[chunks] = off;  // total
    for (uint32_t l = 0; l < nLight; l++)
        lights[l].pdf_power = off > 0.0 ? (float)(emit_lum(lights[l]) / off) : 0.0f;
}
__global__ void k_emit_normalise(uint32_t n, uint32_t chunks, double *cdf, const double *chunk) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double total = chunk[chunks];
    cdf[i] = total > 0.0 ? (cdf[i] + chunk[i / EMIT_CHUNK]) / total : 0.0;
}
void launch_emit_cdf(const float *V, const uint4 *tri, const uint32_t *emit_tri,
                     const uint32_t *emit_light, uint32_t n, DevLight *lights, uint32_t nLight,
                     double *cdf, double *chunk, cudaStream_t s) {
    if (n == 0) return;
    uint32_t chunks = (n + EMIT_CHUNK - 1) / EMIT_CHUNK;
    k_emit_chunks<<<(chunks + 127) / 128, 128, 0, s>>>(V, tri, emit_tri, emit_light, n, lights, cdf, chunk);
    k_emit_offsets<<<1, 1, 0, s>>>(chunks, chunk, lights, nLight);
    k_emit_normalise<<<(n + 255) / 256, 256, 0, s>>>(n, chunks, cdf, chunk);
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

// First node of a captured wave: the wave's first sample index and first frame, which the
// host sets as this node's arguments before every replay (cudaGraphExecKernelNodeSetParams).
__global__ void k_wave_begin(uint64_t base, uint64_t frame, uint64_t *cur) {
    cur[0] = base;
    cur[1] = frame;
}
void launch_wave_begin(uint64_t base, uint64_t frame, uint64_t *cur, cudaStream_t s) {
    k_wave_begin<<<1, 1, 0, s>>>(base, frame, cur);
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
