// wl_disney.cuh - the reference's Disney BSDF, light sampling and tone map on the device.
//
// Restates src/Frontend/Device/{Common,Evaluate,Pdf,Sample,Tonemap}.h in the same expression
// order (so that WL_MATH_STRICT builds are bit-identical to the CPU oracle); the clearcoat
// terms Dr/Fr/Gr that EvalDisneyBSDF computes but never uses (Evaluate.h:165-168) are omitted.
#pragma once
#include "wl_math.cuh"
#include "../../include/wayland_b200.h"

namespace wl {

struct Mat {
    v3 color;
    float metallic, roughness, specular, specular_tint, eta, trans, subsurface, sheen, sheen_tint,
        clearcoat, clearcoat_gloss;
};
WL_HD Mat load_mat(const wl_disney *m) {
    Mat r;
    r.color = v3(m->color[0], m->color[1], m->color[2]);
    r.metallic = m->metallic; r.roughness = m->roughness; r.specular = m->specular;
    r.specular_tint = m->specular_tint; r.eta = m->eta; r.trans = m->trans;
    r.subsurface = m->subsurface; r.sheen = m->sheen; r.sheen_tint = m->sheen_tint;
    r.clearcoat = m->clearcoat; r.clearcoat_gloss = m->clearcoat_gloss;
    return r;
}

// Common.h:102-181
WL_HD void onb(v3 n, v3 &u, v3 &v) {
    float x = n.x, y = n.y, z = n.z;
    float sign = copysignf(1.0f, z);
    float a = -1.0f / (sign + z);
    float b = x * y * a;
    u = v3(1.0f + sign * x * x * a, sign * b, -sign * x);
    v = v3(b, sign + y * y * a, -y);
}
WL_HD float schlick(float u) {
    float m = clampf(1.0f - u, 0.0f, 1.0f);
    float m2 = m * m;
    return m2 * m2 * m;
}
WL_HD float fresnel(float ci, float ct, float eta) {
    const float rs = (ci - ct * eta) / (ci + eta * ct);
    const float rp = (ci * eta - ct) / (ci * eta + ct);
    return 0.5f * (rs * rs + rp * rp);
}
WL_HD float gtr1(float ndh, float a) {
    if (a >= 1.0f) return 1.0f / PI;
    float a2 = a * a;
    float t = 1.0f + (a2 - 1.0f) * ndh * ndh;
    return (a2 - 1.0f) / (PI * m_log(a2) * t);
}
WL_HD float gtr2(float ndh, float a) {
    float a2 = a * a;
    float t = 1.0f + (a2 - 1.0f) * ndh * ndh;
    return a2 / (PI * t * t);
}
WL_HD float smithg(float ndv, float ag) {
    float a = ag * ag;
    float b = ndv * ndv;
    return 1.0f / (ndv + sqrtf(a + b - a * b));
}
WL_HD float lambda_beckmann(v3 w, v3 n) {
    const float alphax = 0.5f;
    float wdn = dot(w, n);
    float abs_tan = fabsf(length(cross(w, n)) / wdn);
    if (isinf(abs_tan)) return 0.0f;
    float a = 1.0f / (alphax * abs_tan);
    if (a >= 1.6f) return 0.0f;
    return (1.0f - 1.259f * a + 0.396f * a * a) / (3.535f * a + 2.181f * a * a);
}
WL_HD v3 ctint_of(v3 cdlin) {
    float cdlum = 0.3f * cdlin.x + 0.6f * cdlin.y + 0.1f * cdlin.z;
    return cdlum > 0.0f ? cdlin / cdlum : v3(1.0f);
}
WL_HD v3 cspec0(const Mat &m, v3 cdlin, v3 ctint) {
    return lerpv(m.specular * 0.08f * lerpv(v3(1.0f), ctint, m.specular_tint), cdlin, m.metallic);
}

// EvalDisneyTransmit, Evaluate.h:10-76
WL_HD v3 eval_transmit(const Mat &m, v3 Ns, v3 V, v3 L, v3 tex) {
    v3 N = Ns;
    v3 cc = tex * m.color;
    float ndl = dot(N, L);
    float ndv = dot(N, V);
    float eta = 1.0f / m.eta;
    if (ndl > 0.0f) {
        eta = 1.0f / eta;
        N = -N;
    }
    if (ndl == 0.0f || ndv == 0.0f) return v3(0.0f);
    float refract = ((1.0f - ndv * ndv) * eta * eta >= 1.0f) ? 1.0f : 0.0f;
    v3 wh = normalize(L + V * eta);
    if (dot(wh, N) < 0.0f) wh = -wh;
    if (dot(L, wh) * dot(V, wh) > 0.0f) return v3(0.0f);
    float sqrt_denom = dot(L, wh) + eta * dot(V, wh);
    float factor = 1.0f / eta;
    v3 Tc = m.trans * cc;
    float gs = 1.0f / (1.0f + lambda_beckmann(V, N) + lambda_beckmann(L, N));
    float a = fmaxf(0.001f, m.roughness);
    float ds = gtr2(dot(N, wh), a);
    float f = fresnel(fabsf(dot(V, wh)), fabsf(dot(L, wh)), eta);
    return (1.0f - refract) * (1.0f - f) * Tc *
           fabsf(ds * gs * eta * eta * fabsf(dot(L, wh)) * fabsf(dot(V, wh)) * factor * factor /
                 (ndl * ndl * sqrt_denom * sqrt_denom));
}

// EvalDisneyBSDF, Evaluate.h:78-191
WL_HD v3 eval_disney(const Mat &m, v3 Ns_, v3 Ng, v3 V, v3 L, v3 tex) {
    v3 cc = tex * m.color;
    v3 Ns = Ns_;
    float ndl = dot(Ns, L);
    float gndl = dot(Ng, L);
    float ndv = dot(Ns, V);
    float gndv = dot(Ng, V);
    float eta = 1.0f / m.eta;
    if (m.trans < 0.1f && (gndl * gndv <= 0.0f || ndl * ndv <= 0.0f)) return v3(0.0f);
    if (m.trans > 0.9f && (gndl * gndv * ndl * ndv <= 0.0f)) return v3(0.0f);
    if (ndl * ndv <= 0.0f) return eval_transmit(m, Ns, V, L, tex);
    if (m.metallic + cc.x + cc.y + cc.z <= 0.0f) return v3(0.0f);
    if (ndl < 0.0f && ndv < 0.0f) {
        Ns = -Ns;
        eta = 1.0f / eta;
        ndl *= -1.0f;
        ndv *= -1.0f;
    }
    v3 H = normalize(L + V);
    float ndh = dot(Ns, H);
    float ldh = dot(L, H);
    float refract = ((1.0f - ndv * ndv) * eta * eta >= 1.0f) ? 1.0f : 0.0f;
    v3 cdlin = cc;
    v3 ctint = ctint_of(cdlin);
    v3 cs0 = cspec0(m, cdlin, ctint);
    v3 csheen = lerpv(v3(1.0f), ctint, m.sheen_tint);
    float fl = schlick(ndl), fv = schlick(ndv);
    float fd90 = 0.5f + 2.0f * ldh * ldh * m.roughness;
    float fd = lerpf(1.0f, fd90, fl) * lerpf(1.0f, fd90, fv);
    float fss90 = ldh * ldh * m.roughness;
    float fss = lerpf(1.0f, fss90, fl) * lerpf(1.0f, fss90, fv);
    float ss = 1.25f * (fss * (1.0f / (ndl + ndv) - 0.5f) + 0.5f);
    float a = fmaxf(0.001f, m.roughness);
    float ds = gtr2(ndh, a);
    float fh = schlick(ldh);
    v3 fs = lerpv(cs0, v3(1.0f), fh);
    float roughg = sqrtf(m.roughness * 0.5f + 0.5f);
    float gs = smithg(ndl, roughg) * smithg(ndv, roughg);
    v3 fsheen = fh * m.sheen * csheen;
    float trans = m.trans;
    float cos_i = fabsf(dot(Ns, V));
    float sin2_i = 1.0f - cos_i * cos_i;
    float sin2_t = eta * eta * sin2_i;
    float cos_t = 1.0f;
    if (sin2_t <= 1.0f) cos_t = sqrtf(1.0f - sin2_t);
    float f = fresnel(cos_i, cos_t, eta);
    v3 out = ((RECIP_PI * lerpf(fd, ss, m.subsurface) * cdlin + fsheen) * (1.0f - m.metallic)) *
             (1.0f - trans * (1.0f - f) * (1.0f - refract));
    if (trans > 0.0f)
        out = out + gs * ds * (1.0f - trans * (1.0f - refract) * (1.0f - f));
    else
        out = out + gs * ds * fs;
    return out;
}

// PdfDisneyBSDF, Pdf.h:42-117
WL_HD float pdf_disney(const Mat &m, v3 Ns_, v3 V, v3 L) {
    float trans_ratio = m.trans;
    v3 Ns = Ns_;
    float eta = m.eta;
    if (dot(Ns, V) < 0.0f) {
        eta = 1.0f / eta;
        Ns = -Ns;
    }
    float ndv = fabsf(dot(V, Ns));
    v3 wh = -normalize(V + L * eta);
    float spec_alpha = m.roughness;
    float cc_alpha = lerpf(0.1f, 0.001f, m.clearcoat_gloss);
    float diffuse_ratio = 0.5f * (1.0f - m.metallic);
    float specular_ratio = 1.0f - diffuse_ratio;
    v3 half = normalize(L + V);
    float cos_theta = fabsf(dot(half, Ns));
    float pdf_gtr2 = gtr2(cos_theta, spec_alpha) * cos_theta;
    float pdf_gtr1 = gtr1(cos_theta, cc_alpha) * cos_theta;
    float ratio = 1.0f / (1.0f + m.clearcoat);
    float pdf_spec = lerpf(pdf_gtr1, pdf_gtr2, ratio) / (4.0f * fabsf(dot(L, half)));
    float pdf_diff = fabsf(dot(L, Ns)) * RECIP_PI;
    float cos_i = fabsf(dot(wh, V));
    float sin2_i = 1.0f - cos_i * cos_i;
    float sin2_t = 1.0f / (eta * eta) * sin2_i;
    float refract_ratio = 0.0f;
    float temp = (1.0f - ndv * ndv) / (eta * eta);
    if (temp < 1.0f) refract_ratio = 1.0f - fresnel(ndv, sqrtf(1.0f - temp), eta);
    float pdf = (diffuse_ratio * pdf_diff + specular_ratio * pdf_spec) * (1.0f - trans_ratio * refract_ratio);
    if (sin2_t <= 1.0f && dot(L, wh) * dot(V, wh) < 0.0f) {
        float sqrt_denom = eta * dot(L, wh) + dot(V, wh);
        float dwh_dwi = fabsf((eta * eta * dot(L, wh)) / (sqrt_denom * sqrt_denom));
        float a = fmaxf(0.001f, m.roughness);
        float ds = gtr2(fabsf(dot(wh, Ns)), a);
        float pdf_trans = ds * fabsf(dot(Ns, wh)) * dwh_dwi;
        pdf += trans_ratio * pdf_trans * refract_ratio;
    }
    cos_i = fabsf(dot(half, V));
    sin2_i = 1.0f - cos_i * cos_i;
    sin2_t = 1.0f / (eta * eta) * sin2_i;
    if (sin2_t > 1.0f)
        pdf += (diffuse_ratio * pdf_diff + specular_ratio * pdf_spec) * trans_ratio * refract_ratio;
    return pdf;
}

// SampleUniformDisk + SampleCosineHemisphere, Sample.h:24-52
WL_HD v3 sample_cosine_hemisphere(v3 n, Rng &rng) {
    v3 x, y;
    onb(n, x, y);
    float r = sqrtf(rng.next());
    float theta = rng.next() * TWO_PI;
    float dx = r * m_cos(theta), dy = r * m_sin(theta);
    float z = sqrtf(1.0f - dx * dx - dy * dy);
    return x * dx + y * dy + n * z;
}

// SampleDisneyBSDF, Sample.h:134-231 (7 uniforms, +2 for the cosine lobe)
WL_HD v3 sample_disney(const Mat &m, v3 Ns_, v3 V, Rng &rng) {
    float r1 = rng.next(), r2 = rng.next(), r3 = rng.next(), r4 = rng.next();
    v3 Ns = Ns_;
    float eta = 1.0f / m.eta;
    if (dot(Ns, V) < 0.0f) {
        eta = 1.0f / eta;
        Ns = -Ns;
    }
    float ndv = fabsf(dot(Ns, V));
    float trans_ratio = m.trans;
    float transprob = rng.next();
    float refractprob = rng.next();
    float probability = rng.next();
    float diffuse_ratio = 0.5f * (1.0f - m.metallic);
    if (transprob < trans_ratio) {
        float refract_ratio = 0.0f;
        float temp = (1.0f - ndv * ndv) * (eta * eta);
        if (temp < 1.0f) refract_ratio = 1.0f - fresnel(ndv, sqrtf(1.0f - temp), eta);
        if (refractprob < refract_ratio) {
            v3 ox, oy;
            onb(Ns, ox, oy);
            float a = m.roughness;
            float phi = r3 * TWO_PI;
            float cos_t = sqrtf((1.0f - r4) / (1.0f + (a * a - 1.0f) * r4));
            float sin_t = sqrtf(1.0f - (cos_t * cos_t));
            float sin_p = m_sin(phi);
            float cos_p = m_cos(phi);
            v3 h(sin_t * cos_p, sin_t * sin_p, cos_t);
            h = h.x * ox + h.y * oy + h.z * Ns;
            if (dot(V, Ns) == 0.0f) return -V;
            float cos_i = dot(h, V);
            float sin2_i = 1.0f - cos_i * cos_i;
            float sin2_t = eta * eta * sin2_i;
            if (sin2_t <= 1.0f) {
                float cos_tt = sqrtf(1.0f - sin2_t);
                v3 L = normalize(eta * -V + (eta * cos_i - cos_tt) * h);
                if (cos_i < 0.0f) {
                    float ldh = dot(L, h);
                    L = L - 2.0f * ldh * h;
                }
                return L;
            }
            return h * 2.0f * dot(h, V) - V;
        }
    }
    v3 ox, oy;
    onb(Ns, ox, oy);
    v3 dir;
    if (probability < diffuse_ratio) {
        dir = sample_cosine_hemisphere(Ns, rng);
    } else {
        float a = m.roughness;
        float phi = r1 * TWO_PI;
        float cos_t = sqrtf((1.0f - r2) / (1.0f + (a * a - 1.0f) * r2));
        float sin_t = sqrtf(1.0f - (cos_t * cos_t));
        float sin_p = m_sin(phi);
        float cos_p = m_cos(phi);
        v3 h(sin_t * cos_p, sin_t * sin_p, cos_t);
        h = h.z * Ns + h.x * ox + h.y * oy;
        dir = 2.0f * dot(V, h) * h - V;
    }
    return dir;
}

// AceApprox, Tonemap.h:34-43 (glm::clamp: min(max(x, 0), 1), NaN preserved)
WL_HD v3 ace(v3 rad) {
    rad = rad * 0.6f;
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    v3 q = (rad * (a * rad + b)) / (rad * (c * rad + d) + e);
    auto gc = [](float x) {
        float t = (x < 0.0f) ? 0.0f : x;
        return (1.0f < t) ? 1.0f : t;
    };
    return v3(gc(q.x), gc(q.y), gc(q.z));
}

}  // namespace wl
