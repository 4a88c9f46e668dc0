// pz_optics.cuh -- optics and spectral helpers (pk.h:165-205, 405-450, 932-1033).
// Written to keep the reference's operation order; units that need bit-exact results
// with the CPU oracle compile them with -fmad=false.
#pragma once
#include "pz_common.cuh"

namespace pz {

// square2triangle, pk.h:165-178
PZ_D float2 square2triangle(float2 s)
{
    if (s.y > s.x) {
        s.x *= 0.5f;
        s.y -= s.x;
    } else {
        s.y *= 0.5f;
        s.x -= s.y;
    }
    return s;
}

// refraction_norm_free, pk.h:181-200 (normal direction defines in/out of the medium)
PZ_D bool refraction_norm_free(float3* wo, float3 wi, float3 n, float eta)
{
    float NoN = dot(n, n);
    float WIoN = dot(wi, n);
    if (WIoN < 0.0f) {
        WIoN = -WIoN;
        n = -n;
        eta = 1.0f / eta;
    }
    float WIoWI = dot(wi, wi);
    float k = NoN * WIoWI * (eta * eta - 1.0f) + WIoN * WIoN;
    if (k < 0.0f) return false;
    *wo = -wi * NoN + (WIoN - sqrtf(k)) * n;
    return true;
}

// reflection, pk.h:202-205
PZ_D float3 reflection(float3 wi, float3 n) { return n * dot(wi, n) * 2.0f / dot(n, n) - wi; }

// fresnel_exact_norm_free, pk.h:427-450
PZ_D float fresnel_exact_norm_free(float3 wi, float3 n, float eta)
{
    float nn = dot(n, n), wiwi = dot(wi, wi), C = dot(n, wi);
    if (C < 0.0f) {
        C = -C;
        n = -n;
        eta = 1.0f / eta;
    }
    float K = nn * wiwi * (eta * eta - 1.0f) + C * C;
    if (K < 0.0f) return 1.0f;
    float G = sqrtf(K);
    float GmC = G - C, GpC = G + C;
    float a = GmC / GpC;
    float b = (C * GpC - nn * wiwi) / (C * GmC + nn * wiwi);
    return 0.5f * (a * a) * (1.0f + b * b);
}

// CIE 2015 10-degree analytic CMFs and the logistic sampling of CMF-y (pk.h:960-1012),
// evaluated with the accurate expf/logf.
PZ_D float asym_gauss(float x, float mean, float sigma, float a)
{
    float denom = sigma + a * (x - mean);
    if (denom < 1.0e-15f) denom = 1.0e-15f;
    if (sigma * 2.0f < denom) denom = sigma * 2.0f;
    float k = (x - mean) / denom;
    return expf(-k * k);
}
PZ_D float cmf_x(float x)
{
    float a = 0.42f * asym_gauss(x, 445.5849609375f, 31.146467208862305f, 0.06435633450746536f);
    float b = 1.16f * asym_gauss(x, 594.5570068359375f, 48.602108001708984f, -0.04772702232003212f);
    return (a + b - a * b * 42.559776306152344f) * 1.0008530432426956f;
}
PZ_D float cmf_y(float x)
{
    return 1.0f * asym_gauss(x, 556.8383178710938f, 66.54190826416016f, -0.026492968201637268f) * 1.004315086937574f;
}
PZ_D float cmf_z(float x)
{
    return 2.146832f * asym_gauss(x, 445.9251708984375f, 30.91781997680664f, 0.08379141241312027f) * 0.9975112815948937f;
}
PZ_D float logistic_pdf(float x, float s)
{
    float k = expf(-fabsf(x) / s);
    return (float)(k / ((1.0 + k) * (1.0 + k) * s));
}
PZ_D float logistic_cdf(float x, float s) { return 1.0f / (1.0f + expf(-x / s)); }
PZ_D float inverse_logistic_cdf(float u, float s)
{
    if (0.99999994f < u) u = 0.99999994f;
    if (u < 1.175494351e-38f) u = 1.175494351e-38f;
    return -s * logf(1.0f / u - 1.0f);
}
PZ_D float cmf_y_pdf(float x)
{
    const float s = 26.879621505737305f;
    return logistic_pdf(x - 554.270751953125f, s) /
           (logistic_cdf(275.729248046875f, s) - logistic_cdf(-164.270751953125f, s));
}
PZ_D float cmf_y_sample(float u)
{
    const float s = 26.879621505737305f;
    float Pa = logistic_cdf(-164.270751953125f, s), Pb = logistic_cdf(275.729248046875f, s);
    return inverse_logistic_cdf(Pa + (Pb - Pa) * u, s) + 554.270751953125f;
}
PZ_D float3 xyz2srgblinear(float3 xyz)
{
    return mk3(dot(mk3(3.2406f, -1.5372f, -0.4986f), xyz), dot(mk3(-0.9689f, 1.8758f, 0.0415f), xyz),
               dot(mk3(0.0557f, -0.204f, 1.057f), xyz));
}
constexpr float kIntegralCmfY = 118.51810464018001f;

// spectral RGB weight of a wavelength (pk.h / main_gpu.cu:356-361 and :473-478)
PZ_D float3 lambda_to_srgb(float lambda)
{
    float3 xyz = mk3(cmf_x(lambda) / kIntegralCmfY, cmf_y(lambda) / kIntegralCmfY, cmf_z(lambda) / kIntegralCmfY);
    return xyz2srgblinear(xyz);
}

}  // namespace pz
