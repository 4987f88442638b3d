// sfp_gk_rules.h -- generated by sfparticles_b200/qed/gauss_kronrod.py; do not edit.
// Gauss-Kronrod rules: xgk (non-negative nodes, decreasing, centre last), wgk
// (Kronrod weights), wg (Gauss weights of the nodes xgk[1], xgk[3], ...),
// as accessors usable in host and device code.
#pragma once
#ifndef SFP_HD
#if defined(__CUDACC__)
#define SFP_HD __host__ __device__ inline
#else
#define SFP_HD inline
#endif
#endif

namespace sfp_gk {

SFP_HD double xgk15(int i) {
    constexpr double v[8] = {0x1.fba009d4d09b1p-1, 0x1.e5f178e7c6229p-1, 0x1.bacf827b9bb3ep-1, 0x1.7ba9f9be3a1d6p-1, 0x1.2c13a049dfa24p-1, 0x1.9f95df119fd62p-2, 0x1.a98b2892e0c77p-3, 0x0.0p+0};
    return v[i];
}
SFP_HD double wgk15(int i) {
    constexpr double v[8] = {0x1.77c5b67d57470p-6, 0x1.026cdaa7b61c4p-4, 0x1.ad384a34814c6p-4, 0x1.200ed0f46e8c1p-3, 0x1.5a1f266e47d5cp-3, 0x1.85d6861c80eb1p-3, 0x1.a2adbcbec9cd8p-3, 0x1.ad04f9087090fp-3};
    return v[i];
}
SFP_HD double wg15(int i) {
    constexpr double v[4] = {0x1.092f69f826d57p-3, 0x1.1e6b1713d8644p-2, 0x1.86fe74ee32b3dp-2, 0x1.abfd7e03c2fa6p-2};
    return v[i];
}

SFP_HD double xgk21(int i) {
    constexpr double v[11] = {0x1.fdc6c69272ae5p-1, 0x1.f2a3e062af2d8p-1, 0x1.dc3d9a4b011c6p-1, 0x1.bae995e9cb2f3p-1, 0x1.8fc7574fa6c62p-1, 0x1.5bdb9228de198p-1, 0x1.2021b401fc120p-1, 0x1.bbcc009016adcp-2, 0x1.2d755295ea137p-2, 0x1.30e507891e27ap-3, 0x0.0p+0};
    return v[i];
}
SFP_HD double wgk21(int i) {
    constexpr double v[11] = {0x1.7f35bdbca883fp-7, 0x1.0ab76a4a94042p-5, 0x1.c08f7021999a2p-5, 0x1.335ccd53722e5p-4, 0x1.7d711dddcb389p-4, 0x1.c00cbfda8818fp-4, 0x1.f9d2b8f5d2ddep-4, 0x1.13e26d16948d4p-3, 0x1.2467b616c0e05p-3, 0x1.2e91d6ff21eb5p-3, 0x1.321082b7cd10fp-3};
    return v[i];
}
SFP_HD double wg21(int i) {
    constexpr double v[5] = {0x1.1115f8b62dc1fp-4, 0x1.32138c878efe5p-3, 0x1.c0b059d00bc31p-3, 0x1.13baa7a559bfep-2, 0x1.2e9de7014d6efp-2};
    return v[i];
}

}  // namespace sfp_gk
