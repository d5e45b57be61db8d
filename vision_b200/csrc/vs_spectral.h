// Spectral helpers shared by the host (scene build, light power) and the
// kernels: 5-nm CIE/D65 lookup tables built the way the reference's SPD class
// builds them, the sigmoid-polynomial RGB uplift evaluator and Planck's law.
#pragma once

#include "vs_math.h"

namespace vs {

constexpr float kLambdaMin = 360.0f;
constexpr float kLambdaMax = 830.0f;
constexpr int kCieSamples = 471;  // 1 nm, 360..830
constexpr int kSpd5Count = 94;    // reference downsamples every 5th sample, 360..825 nm

// Piecewise-linear SPD lookup with the reference's sample spacing
// (src/base/color/spd.cpp:67-86): the spacing is 471 / n (not 5 nm), the index
// is clamped to n - 2 and the weight is fract(t).
VS_HD float spd_eval(const float *f, int n, float lambda) {
    float interval = static_cast<float>(kCieSamples) / static_cast<float>(n);
    float t = (clampf(lambda, kLambdaMin, kLambdaMax) - kLambdaMin) / interval;
    uint32_t sample_count = static_cast<uint32_t>((kLambdaMax - kLambdaMin) / interval) + 1u;
    uint32_t i = static_cast<uint32_t>(fminf(t, static_cast<float>(sample_count - 2u)));
    float fr = t - floorf(t);
    float l = f[i], r = f[i + 1];
    return l + fr * (r - l);
}

// Sigmoid of the RGB uplift (src/render_core/spectra/hero.cpp:27-49).
VS_HD float sigmoid_poly(float c0, float c1, float c2, float lambda) {
    float x = fmaf(fmaf(c0, lambda, c1), lambda, c2);
    if (std::isinf(x)) return x > 0.0f ? 1.0f : 0.0f;
    return 0.5f * fmaf(x, 1.0f / sqrtf(fmaf(x, x, 1.0f)), 1.0f);
}

// Planck's law in W / (m^2 sr m), lambda in nm (src/math/optics.h:82-90).
VS_HD float planck(float lambda_nm, float T) {
    const float c = 299792458.0f;
    const float h = 6.62606957e-34f;
    const float kb = 1.3806488e-23f;
    float l = lambda_nm * 1e-9f;
    float l2 = l * l;
    float l5 = l2 * l2 * l;
    return (2.0f * h * c * c) / (l5 * (expf((h * c) / (l * kb * T)) - 1.0f));
}

// Wien's displacement: wavelength of the Planck peak, in nm.
VS_HD float planck_peak_nm(float T) { return 2.8977721e-3f / T * 1e9f; }

// Hero-wavelength importance density (src/render_core/spectra/hero.cpp:15-25).
VS_HD float sample_visible_wavelength(float u) {
    return 538.0f - 138.888889f * atanhf(0.85691062f - 1.82750197f * u);
}
VS_HD float visible_wavelength_pdf(float lambda) {
    return 0.0039398042f / sqr(coshf(0.0072f * (lambda - 538.0f)));
}

// XYZ -> linear sRGB (src/base/color/cie.h:414-421).
VS_HD f3 xyz_to_linear_srgb(f3 xyz) {
    return {3.240479f * xyz.x - 1.537150f * xyz.y - 0.498535f * xyz.z,
            -0.969256f * xyz.x + 1.875991f * xyz.y + 0.041556f * xyz.z,
            0.055648f * xyz.x - 0.204043f * xyz.y + 1.057311f * xyz.z};
}
VS_HD float linear_srgb_to_y(f3 rgb) {
    return 0.212671f * rgb.x + 0.715160f * rgb.y + 0.072169f * rgb.z;
}

}  // namespace vs
