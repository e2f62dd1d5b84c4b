// Generated by eu3d_b200/codegen_mech.py from the H2_JA919 mechanism and
// thermo.dat tables (do not edit).  Specialised rate evaluation for that
// mechanism; see the generator's docstring for the formulas.
#pragma once

#include "common.cuh"

namespace eu3d {
namespace h2ja919 {

// tables this code was generated from (compared at handle creation)
constexpr double K_STOI_F[171] = {0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+1, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0x1.0000000000000p+1, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+1, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
constexpr double K_STOI_B[171] = {0x1.0000000000000p+0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0x1.0000000000000p+1, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0x1.0000000000000p+1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
constexpr double K_TB[171] = {0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.8000000000000p+2, 0x1.8000000000000p+2, 0x1.4000000000000p+2, 0x1.0000000000000p+4, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.e000000000000p+3, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+1, 0x1.0000000000000p+0, 0x1.0000000000000p+1, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0x1.0000000000000p+0};
constexpr double K_AF[19] = {0x1.6bcc41e900000p+46, 0x1.d8efef4880000p+47, 0x1.0c388d0000000p+34, 0x1.402462f600000p+44, 0x1.6eb550c600000p+42, 0x1.2a27d53bc0487p+74, 0x1.1c37937e08000p+59, 0x1.aa535d3d0c000p+55, 0x1.dd7c1681d0000p+50, 0x1.b48eb57e00000p+45, 0x1.fd51291300000p+46, 0x1.2309ce5400000p+43, 0x1.b48eb57e00000p+43, 0x1.d1a94a2000000p+42, 0x1.d1a94a2000000p+40, 0x1.45f680b000000p+40, 0x1.977420dc00000p+43, 0x1.6311155200000p+42, 0x1.aa535d3d0c000p+56};
constexpr double K_BF[19] = {0.0, 0.0, 0x1.0000000000000p+0, 0.0, 0.0, (-0x1.0000000000000p+1), (-0x1.0000000000000p+0), (-0x1.3333333333333p-1), 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
constexpr double K_EAF[19] = {0x1.b5be07fcb923ap+15, 0x1.06a537e90ff97p+14, 0x1.1647837b4a234p+13, 0x1.420d8e8a71de7p+12, 0x1.10a6b1c432ca5p+10, 0.0, 0.0, 0.0, (-0x1.f446e2eb1c433p+9), (-0x1.c23fcd35a8588p+10), 0x1.0e25c5d638866p+10, 0x1.0e25c5d638866p+10, 0x1.db42b367a0f91p+9, 0.0, 0.0, 0x1.c23fcd35a8588p+11, 0x1.9038b6ae7d567p+12, 0x1.65b3212d77319p+10, 0x1.63aa6b923a29cp+15};
constexpr double K_C0[81] = {0.0, (-0x1.f119c7e28240bp+12), (-0x1.346f377318fc5p+15), (-0x1.f3b6f9b13165dp+10), (-0x1.0b9f44b5dcc64p+15), 0x1.3e9e76d5cfaadp+15, (-0x1.6a7b55f6fd220p+16), (-0x1.28d4d34d6a162p+16), 0x1.595edc21187e8p+14, 0.0, 0x1.416f80b09487ep+7, 0x1.1fc95b6805a2dp+9, 0x1.740164ef6de18p+6, 0x1.e4b3398e97072p+8, (-0x1.907594d0dcfccp+9), 0x1.872fe58a32f45p+10, 0x1.4c58921ccd962p+10, (-0x1.7dd89f623076cp+8), 0x1.4000000000000p+1, 0x1.f75a9da7bd962p+0, 0x1.dd129dab3af08p-1, 0x1.86826431358abp+1, 0x1.1e7780995c4bdp+0, 0x1.06ded6bfeabc2p+3, (-0x1.7e7e52abc9720p+2), (-0x1.2b5a54345fae1p+2), 0x1.854b95d594c77p+2, 0.0, 0x1.09ba43524e224p-10, 0x1.d9590385a8417p-8, 0x1.90f4f914b843ep-10, 0x1.196781dbc322fp-8, (-0x1.a00f5e57224a9p-7), 0x1.0bf07bef07e1dp-5, 0x1.9af6123d5cbe6p-6, (-0x1.178a7f32adaccp-7), 0.0, (-0x1.2a132ab53fcefp-20), (-0x1.ecc02cd2de9f9p-18), (-0x1.a7d84ef8ef49fp-19), (-0x1.6f05661ee4981p-21), 0x1.2634c3b74493ep-16, (-0x1.49db350f66c83p-15), (-0x1.f86a684e1dea7p-16), 0x1.d09c33b406855p-17, 0.0, 0x1.664dc37a8c93ap-31, 0x1.54820c03e216fp-28, 0x1.c7abe45c93c67p-29, (-0x1.16171913542eap-29), (-0x1.9d4cb55199da9p-27), 0x1.af16365a726fdp-26, 0x1.45a95f43bda8ep-26, (-0x1.4abd6047b3e3cp-27), 0.0, (-0x1.64dc4dce22bf2p-43), (-0x1.7850316ebe98cp-40), (-0x1.40887fc624544p-40), 0x1.2476b94b5d0c9p-40, 0x1.da045b502c793p-39, (-0x1.c6efe6f8eebcbp-38), (-0x1.53c7bcb8b40e2p-38), 0x1.629df8198e88ap-39, 0x1.8e06d50092ccfp+14, 0x1.bbce7f5ad96a7p+14, (-0x1.021f7c779a6b5p+15), 0x1.75e6db035bd51p+11, (-0x1.a7ee8e4b87bddp+11), 0x1.4f4f82602c908p+11, (-0x1.85b0306a2b170p+14), (-0x1.6f159d883ba34p+12), 0x1.636c4c8bc9cd4p+9, (-0x1.c9673ad546a18p-2), 0x1.0cef8c8a926aap+3, 0x1.13df77f27fe4cp+4, 0x1.2b24a1953b910p+2, 0x1.27f3b0b6ec90bp+4, (-0x1.e701974f118b1p+4), 0x1.d62c86f6ffa64p+5, 0x1.9f7cf8c9aad96p+5, (-0x1.58523a0991235p+3)};
constexpr double K_C1[81] = {0x1.e64d4bf0995abp+5, 0x1.ff87035a85879p+17, 0x1.f95b83126e979p+19, 0x1.f0c62c20c49bap+19, (-0x1.face60b439581p+19), 0x1.11d599a1cac08p+19, 0x1.6ba1406e978d5p+20, (-0x1.ba0edb9581062p+20), 0x1.1ef80cfdf3b64p+19, (-0x1.749a91a0adb35p-3), (-0x1.6cefa459103c9p+9), (-0x1.2d965a9eb2075p+11), (-0x1.39bea2014727ep+11), 0x1.251a91ab8e8eap+11, (-0x1.a29342bb66730p+9), (-0x1.432d2602c9082p+12), 0x1.3633128e0c9dap+12, (-0x1.17e7f867f0aa2p+11), 0x1.4006f0d98b3afp+1, 0x1.a89943c8d79fcp+1, 0x1.2959e1076c5afp+2, 0x1.47758527c79a3p+2, 0x1.d1d9f56e1a7eap+0, 0x1.7cd8beb74f25fp+1, 0x1.69068d17ab177p+3, (-0x1.0a1c9b1edd6e6p+0), 0x1.8448e56199222p+2, (-0x1.076441fdd206cp-23), (-0x1.c0ee31b1f2734p-12), 0x1.2c6ab38ac7604p-9, 0x1.11bdc1a276f27p-13, 0x1.4c5bcf9aa0723p-10, 0x1.48450422d75b8p-10, (-0x1.515296b6985f4p-14), 0x1.2ada98cd1ee1dp-8, (-0x1.41e576be829a1p-11), 0x1.4858e6f97727fp-35, 0x1.bd00e7a587463p-24, (-0x1.6f0caec06cb5ep-21), (-0x1.63cf1626e78d2p-24), (-0x1.d5e24f4c55a11p-23), (-0x1.91a8060fc0cc0p-22), (-0x1.38655d2945373p-26), (-0x1.1d0a6cf1d43c0p-20), 0x1.405cf082ec2ddp-23, (-0x1.99d85e45f4e6fp-48), (-0x1.4c14b00ee3b1bp-37), 0x1.9e949adad1c37p-34, 0x1.60fba49bca098p-36, 0x1.694b4e970430ep-36, 0x1.0518752509928p-34, 0x1.e8decf9673d0bp-38, 0x1.f762e3002e92cp-34, (-0x1.5250f8b15de24p-36), 0x1.929b476864976p-62, 0x1.3a2cef3ab0f03p-52, (-0x1.5b7d382eb9503p-48), (-0x1.c0c5da9edbba5p-50), (-0x1.d8523b5720180p-51), (-0x1.03e94c0ab008ap-48), (-0x1.164e393d55d7bp-51), (-0x1.5737068b814bfp-48), 0x1.32166731f41f3p-50, 0x1.8e0b74b72c519p+14, 0x1.09088faacd9e8p+15, (-0x1.b096ebb44e50cp+13), 0x1.3b919bb59ddc2p+14, (-0x1.07e86fe9b7bf2p+14), 0x1.4dbd30c88a47fp+12, 0x1.bb3415421c044p+13, (-0x1.f420b0068db8cp+14), 0x1.9100d54c985f0p+13, (-0x1.caf2c902345a2p-2), (-0x1.55fea93dd171dp-1), (-0x1.fe99fc3545313p+2), (-0x1.60690c8e58c8cp+3), 0x1.1631d3fd6da98p+4, (-0x1.19f4860ca78bdp+1), (-0x1.7411861f6951dp+5), 0x1.45591b59f899ep+5, (-0x1.fbb98d0f1ca88p+3)};
constexpr double K_MW[9] = {0x1.02085b18548aap+0, 0x1.fffb15b573eabp+3, 0x1.203e963dc486bp+4, 0x1.101e108c3f3e0p+4, 0x1.fffb15b573eabp+4, 0x1.02085b18548aap+1, 0x1.101e108c3f3e0p+5, 0x1.080dcdb37c99bp+5, 0x1.c036e2eb1c433p+4};

// H/R, S/R of species s at p (both NASA-9 ranges as literals)
template <int S> __device__ __forceinline__ double h_r_spec(const TPow &p);
template <int S> __device__ __forceinline__ double s_r_spec(const TPow &p);
template <int S> __device__ __forceinline__ double cp_r_spec(const TPow &p);
template <> __device__ __forceinline__ double h_r_spec<0>(const TPow &p)
{
    return p.hi ? (-0x1.e64d4bf0995abp+5 * p.tm1 + (-0x1.749a91a0adb35p-3) * p.lnT + 0x1.4006f0d98b3afp+1 * p.T + (-0x1.076441fdd206cp-23) * p.t2 * 0.5 + 0x1.4858e6f97727fp-35 * p.t3 * (1.0 / 3.0) + (-0x1.99d85e45f4e6fp-48) * p.t4 * 0.25 + 0x1.929b476864976p-62 * p.t5 * 0.2 + (p.rb ? 0x1.8e0b74b72c519p+14 : 0x1.8e06d50092ccfp+14)) : (-0.0 * p.tm1 + 0.0 * p.lnT + 0x1.4000000000000p+1 * p.T + 0.0 * p.t2 * 0.5 + 0.0 * p.t3 * (1.0 / 3.0) + 0.0 * p.t4 * 0.25 + 0.0 * p.t5 * 0.2 + 0x1.8e06d50092ccfp+14);
}
template <> __device__ __forceinline__ double s_r_spec<0>(const TPow &p)
{
    return p.hi ? (-0x1.e64d4bf0995abp+5 * p.tm2 * 0.5 - (-0x1.749a91a0adb35p-3) * p.tm1 + 0x1.4006f0d98b3afp+1 * p.lnT + (-0x1.076441fdd206cp-23) * p.T + 0x1.4858e6f97727fp-35 * p.t2 * 0.5 + (-0x1.99d85e45f4e6fp-48) * p.t3 * (1.0 / 3.0) + 0x1.929b476864976p-62 * p.t4 * 0.25 + (p.rb ? (-0x1.caf2c902345a2p-2) : (-0x1.c9673ad546a18p-2))) : (-0.0 * p.tm2 * 0.5 - 0.0 * p.tm1 + 0x1.4000000000000p+1 * p.lnT + 0.0 * p.T + 0.0 * p.t2 * 0.5 + 0.0 * p.t3 * (1.0 / 3.0) + 0.0 * p.t4 * 0.25 + (-0x1.c9673ad546a18p-2));
}
template <> __device__ __forceinline__ double cp_r_spec<0>(const TPow &p)
{
    return p.hi ? (0x1.e64d4bf0995abp+5 * p.tm2 + (-0x1.749a91a0adb35p-3) * p.tm1 + 0x1.4006f0d98b3afp+1 + (-0x1.076441fdd206cp-23) * p.T + 0x1.4858e6f97727fp-35 * p.t2 + (-0x1.99d85e45f4e6fp-48) * p.t3 + 0x1.929b476864976p-62 * p.t4) : (0.0 * p.tm2 + 0.0 * p.tm1 + 0x1.4000000000000p+1 + 0.0 * p.T + 0.0 * p.t2 + 0.0 * p.t3 + 0.0 * p.t4);
}
template <> __device__ __forceinline__ double h_r_spec<1>(const TPow &p)
{
    return p.hi ? (-0x1.ff87035a85879p+17 * p.tm1 + (-0x1.6cefa459103c9p+9) * p.lnT + 0x1.a89943c8d79fcp+1 * p.T + (-0x1.c0ee31b1f2734p-12) * p.t2 * 0.5 + 0x1.bd00e7a587463p-24 * p.t3 * (1.0 / 3.0) + (-0x1.4c14b00ee3b1bp-37) * p.t4 * 0.25 + 0x1.3a2cef3ab0f03p-52 * p.t5 * 0.2 + (p.rb ? 0x1.09088faacd9e8p+15 : 0x1.bbce7f5ad96a7p+14)) : (-(-0x1.f119c7e28240bp+12) * p.tm1 + 0x1.416f80b09487ep+7 * p.lnT + 0x1.f75a9da7bd962p+0 * p.T + 0x1.09ba43524e224p-10 * p.t2 * 0.5 + (-0x1.2a132ab53fcefp-20) * p.t3 * (1.0 / 3.0) + 0x1.664dc37a8c93ap-31 * p.t4 * 0.25 + (-0x1.64dc4dce22bf2p-43) * p.t5 * 0.2 + 0x1.bbce7f5ad96a7p+14);
}
template <> __device__ __forceinline__ double s_r_spec<1>(const TPow &p)
{
    return p.hi ? (-0x1.ff87035a85879p+17 * p.tm2 * 0.5 - (-0x1.6cefa459103c9p+9) * p.tm1 + 0x1.a89943c8d79fcp+1 * p.lnT + (-0x1.c0ee31b1f2734p-12) * p.T + 0x1.bd00e7a587463p-24 * p.t2 * 0.5 + (-0x1.4c14b00ee3b1bp-37) * p.t3 * (1.0 / 3.0) + 0x1.3a2cef3ab0f03p-52 * p.t4 * 0.25 + (p.rb ? (-0x1.55fea93dd171dp-1) : 0x1.0cef8c8a926aap+3)) : (-(-0x1.f119c7e28240bp+12) * p.tm2 * 0.5 - 0x1.416f80b09487ep+7 * p.tm1 + 0x1.f75a9da7bd962p+0 * p.lnT + 0x1.09ba43524e224p-10 * p.T + (-0x1.2a132ab53fcefp-20) * p.t2 * 0.5 + 0x1.664dc37a8c93ap-31 * p.t3 * (1.0 / 3.0) + (-0x1.64dc4dce22bf2p-43) * p.t4 * 0.25 + 0x1.0cef8c8a926aap+3);
}
template <> __device__ __forceinline__ double cp_r_spec<1>(const TPow &p)
{
    return p.hi ? (0x1.ff87035a85879p+17 * p.tm2 + (-0x1.6cefa459103c9p+9) * p.tm1 + 0x1.a89943c8d79fcp+1 + (-0x1.c0ee31b1f2734p-12) * p.T + 0x1.bd00e7a587463p-24 * p.t2 + (-0x1.4c14b00ee3b1bp-37) * p.t3 + 0x1.3a2cef3ab0f03p-52 * p.t4) : ((-0x1.f119c7e28240bp+12) * p.tm2 + 0x1.416f80b09487ep+7 * p.tm1 + 0x1.f75a9da7bd962p+0 + 0x1.09ba43524e224p-10 * p.T + (-0x1.2a132ab53fcefp-20) * p.t2 + 0x1.664dc37a8c93ap-31 * p.t3 + (-0x1.64dc4dce22bf2p-43) * p.t4);
}
template <> __device__ __forceinline__ double h_r_spec<2>(const TPow &p)
{
    return p.hi ? (-0x1.f95b83126e979p+19 * p.tm1 + (-0x1.2d965a9eb2075p+11) * p.lnT + 0x1.2959e1076c5afp+2 * p.T + 0x1.2c6ab38ac7604p-9 * p.t2 * 0.5 + (-0x1.6f0caec06cb5ep-21) * p.t3 * (1.0 / 3.0) + 0x1.9e949adad1c37p-34 * p.t4 * 0.25 + (-0x1.5b7d382eb9503p-48) * p.t5 * 0.2 + (p.rb ? (-0x1.b096ebb44e50cp+13) : (-0x1.021f7c779a6b5p+15))) : (-(-0x1.346f377318fc5p+15) * p.tm1 + 0x1.1fc95b6805a2dp+9 * p.lnT + 0x1.dd129dab3af08p-1 * p.T + 0x1.d9590385a8417p-8 * p.t2 * 0.5 + (-0x1.ecc02cd2de9f9p-18) * p.t3 * (1.0 / 3.0) + 0x1.54820c03e216fp-28 * p.t4 * 0.25 + (-0x1.7850316ebe98cp-40) * p.t5 * 0.2 + (-0x1.021f7c779a6b5p+15));
}
template <> __device__ __forceinline__ double s_r_spec<2>(const TPow &p)
{
    return p.hi ? (-0x1.f95b83126e979p+19 * p.tm2 * 0.5 - (-0x1.2d965a9eb2075p+11) * p.tm1 + 0x1.2959e1076c5afp+2 * p.lnT + 0x1.2c6ab38ac7604p-9 * p.T + (-0x1.6f0caec06cb5ep-21) * p.t2 * 0.5 + 0x1.9e949adad1c37p-34 * p.t3 * (1.0 / 3.0) + (-0x1.5b7d382eb9503p-48) * p.t4 * 0.25 + (p.rb ? (-0x1.fe99fc3545313p+2) : 0x1.13df77f27fe4cp+4)) : (-(-0x1.346f377318fc5p+15) * p.tm2 * 0.5 - 0x1.1fc95b6805a2dp+9 * p.tm1 + 0x1.dd129dab3af08p-1 * p.lnT + 0x1.d9590385a8417p-8 * p.T + (-0x1.ecc02cd2de9f9p-18) * p.t2 * 0.5 + 0x1.54820c03e216fp-28 * p.t3 * (1.0 / 3.0) + (-0x1.7850316ebe98cp-40) * p.t4 * 0.25 + 0x1.13df77f27fe4cp+4);
}
template <> __device__ __forceinline__ double cp_r_spec<2>(const TPow &p)
{
    return p.hi ? (0x1.f95b83126e979p+19 * p.tm2 + (-0x1.2d965a9eb2075p+11) * p.tm1 + 0x1.2959e1076c5afp+2 + 0x1.2c6ab38ac7604p-9 * p.T + (-0x1.6f0caec06cb5ep-21) * p.t2 + 0x1.9e949adad1c37p-34 * p.t3 + (-0x1.5b7d382eb9503p-48) * p.t4) : ((-0x1.346f377318fc5p+15) * p.tm2 + 0x1.1fc95b6805a2dp+9 * p.tm1 + 0x1.dd129dab3af08p-1 + 0x1.d9590385a8417p-8 * p.T + (-0x1.ecc02cd2de9f9p-18) * p.t2 + 0x1.54820c03e216fp-28 * p.t3 + (-0x1.7850316ebe98cp-40) * p.t4);
}
template <> __device__ __forceinline__ double h_r_spec<3>(const TPow &p)
{
    return p.hi ? (-0x1.f0c62c20c49bap+19 * p.tm1 + (-0x1.39bea2014727ep+11) * p.lnT + 0x1.47758527c79a3p+2 * p.T + 0x1.11bdc1a276f27p-13 * p.t2 * 0.5 + (-0x1.63cf1626e78d2p-24) * p.t3 * (1.0 / 3.0) + 0x1.60fba49bca098p-36 * p.t4 * 0.25 + (-0x1.c0c5da9edbba5p-50) * p.t5 * 0.2 + (p.rb ? 0x1.3b919bb59ddc2p+14 : 0x1.75e6db035bd51p+11)) : (-(-0x1.f3b6f9b13165dp+10) * p.tm1 + 0x1.740164ef6de18p+6 * p.lnT + 0x1.86826431358abp+1 * p.T + 0x1.90f4f914b843ep-10 * p.t2 * 0.5 + (-0x1.a7d84ef8ef49fp-19) * p.t3 * (1.0 / 3.0) + 0x1.c7abe45c93c67p-29 * p.t4 * 0.25 + (-0x1.40887fc624544p-40) * p.t5 * 0.2 + 0x1.75e6db035bd51p+11);
}
template <> __device__ __forceinline__ double s_r_spec<3>(const TPow &p)
{
    return p.hi ? (-0x1.f0c62c20c49bap+19 * p.tm2 * 0.5 - (-0x1.39bea2014727ep+11) * p.tm1 + 0x1.47758527c79a3p+2 * p.lnT + 0x1.11bdc1a276f27p-13 * p.T + (-0x1.63cf1626e78d2p-24) * p.t2 * 0.5 + 0x1.60fba49bca098p-36 * p.t3 * (1.0 / 3.0) + (-0x1.c0c5da9edbba5p-50) * p.t4 * 0.25 + (p.rb ? (-0x1.60690c8e58c8cp+3) : 0x1.2b24a1953b910p+2)) : (-(-0x1.f3b6f9b13165dp+10) * p.tm2 * 0.5 - 0x1.740164ef6de18p+6 * p.tm1 + 0x1.86826431358abp+1 * p.lnT + 0x1.90f4f914b843ep-10 * p.T + (-0x1.a7d84ef8ef49fp-19) * p.t2 * 0.5 + 0x1.c7abe45c93c67p-29 * p.t3 * (1.0 / 3.0) + (-0x1.40887fc624544p-40) * p.t4 * 0.25 + 0x1.2b24a1953b910p+2);
}
template <> __device__ __forceinline__ double cp_r_spec<3>(const TPow &p)
{
    return p.hi ? (0x1.f0c62c20c49bap+19 * p.tm2 + (-0x1.39bea2014727ep+11) * p.tm1 + 0x1.47758527c79a3p+2 + 0x1.11bdc1a276f27p-13 * p.T + (-0x1.63cf1626e78d2p-24) * p.t2 + 0x1.60fba49bca098p-36 * p.t3 + (-0x1.c0c5da9edbba5p-50) * p.t4) : ((-0x1.f3b6f9b13165dp+10) * p.tm2 + 0x1.740164ef6de18p+6 * p.tm1 + 0x1.86826431358abp+1 + 0x1.90f4f914b843ep-10 * p.T + (-0x1.a7d84ef8ef49fp-19) * p.t2 + 0x1.c7abe45c93c67p-29 * p.t3 + (-0x1.40887fc624544p-40) * p.t4);
}
template <> __device__ __forceinline__ double h_r_spec<4>(const TPow &p)
{
    return p.hi ? (-(-0x1.face60b439581p+19) * p.tm1 + 0x1.251a91ab8e8eap+11 * p.lnT + 0x1.d1d9f56e1a7eap+0 * p.T + 0x1.4c5bcf9aa0723p-10 * p.t2 * 0.5 + (-0x1.d5e24f4c55a11p-23) * p.t3 * (1.0 / 3.0) + 0x1.694b4e970430ep-36 * p.t4 * 0.25 + (-0x1.d8523b5720180p-51) * p.t5 * 0.2 + (p.rb ? (-0x1.07e86fe9b7bf2p+14) : (-0x1.a7ee8e4b87bddp+11))) : (-(-0x1.0b9f44b5dcc64p+15) * p.tm1 + 0x1.e4b3398e97072p+8 * p.lnT + 0x1.1e7780995c4bdp+0 * p.T + 0x1.196781dbc322fp-8 * p.t2 * 0.5 + (-0x1.6f05661ee4981p-21) * p.t3 * (1.0 / 3.0) + (-0x1.16171913542eap-29) * p.t4 * 0.25 + 0x1.2476b94b5d0c9p-40 * p.t5 * 0.2 + (-0x1.a7ee8e4b87bddp+11));
}
template <> __device__ __forceinline__ double s_r_spec<4>(const TPow &p)
{
    return p.hi ? (-(-0x1.face60b439581p+19) * p.tm2 * 0.5 - 0x1.251a91ab8e8eap+11 * p.tm1 + 0x1.d1d9f56e1a7eap+0 * p.lnT + 0x1.4c5bcf9aa0723p-10 * p.T + (-0x1.d5e24f4c55a11p-23) * p.t2 * 0.5 + 0x1.694b4e970430ep-36 * p.t3 * (1.0 / 3.0) + (-0x1.d8523b5720180p-51) * p.t4 * 0.25 + (p.rb ? 0x1.1631d3fd6da98p+4 : 0x1.27f3b0b6ec90bp+4)) : (-(-0x1.0b9f44b5dcc64p+15) * p.tm2 * 0.5 - 0x1.e4b3398e97072p+8 * p.tm1 + 0x1.1e7780995c4bdp+0 * p.lnT + 0x1.196781dbc322fp-8 * p.T + (-0x1.6f05661ee4981p-21) * p.t2 * 0.5 + (-0x1.16171913542eap-29) * p.t3 * (1.0 / 3.0) + 0x1.2476b94b5d0c9p-40 * p.t4 * 0.25 + 0x1.27f3b0b6ec90bp+4);
}
template <> __device__ __forceinline__ double cp_r_spec<4>(const TPow &p)
{
    return p.hi ? ((-0x1.face60b439581p+19) * p.tm2 + 0x1.251a91ab8e8eap+11 * p.tm1 + 0x1.d1d9f56e1a7eap+0 + 0x1.4c5bcf9aa0723p-10 * p.T + (-0x1.d5e24f4c55a11p-23) * p.t2 + 0x1.694b4e970430ep-36 * p.t3 + (-0x1.d8523b5720180p-51) * p.t4) : ((-0x1.0b9f44b5dcc64p+15) * p.tm2 + 0x1.e4b3398e97072p+8 * p.tm1 + 0x1.1e7780995c4bdp+0 + 0x1.196781dbc322fp-8 * p.T + (-0x1.6f05661ee4981p-21) * p.t2 + (-0x1.16171913542eap-29) * p.t3 + 0x1.2476b94b5d0c9p-40 * p.t4);
}
template <> __device__ __forceinline__ double h_r_spec<5>(const TPow &p)
{
    return p.hi ? (-0x1.11d599a1cac08p+19 * p.tm1 + (-0x1.a29342bb66730p+9) * p.lnT + 0x1.7cd8beb74f25fp+1 * p.T + 0x1.48450422d75b8p-10 * p.t2 * 0.5 + (-0x1.91a8060fc0cc0p-22) * p.t3 * (1.0 / 3.0) + 0x1.0518752509928p-34 * p.t4 * 0.25 + (-0x1.03e94c0ab008ap-48) * p.t5 * 0.2 + (p.rb ? 0x1.4dbd30c88a47fp+12 : 0x1.4f4f82602c908p+11)) : (-0x1.3e9e76d5cfaadp+15 * p.tm1 + (-0x1.907594d0dcfccp+9) * p.lnT + 0x1.06ded6bfeabc2p+3 * p.T + (-0x1.a00f5e57224a9p-7) * p.t2 * 0.5 + 0x1.2634c3b74493ep-16 * p.t3 * (1.0 / 3.0) + (-0x1.9d4cb55199da9p-27) * p.t4 * 0.25 + 0x1.da045b502c793p-39 * p.t5 * 0.2 + 0x1.4f4f82602c908p+11);
}
template <> __device__ __forceinline__ double s_r_spec<5>(const TPow &p)
{
    return p.hi ? (-0x1.11d599a1cac08p+19 * p.tm2 * 0.5 - (-0x1.a29342bb66730p+9) * p.tm1 + 0x1.7cd8beb74f25fp+1 * p.lnT + 0x1.48450422d75b8p-10 * p.T + (-0x1.91a8060fc0cc0p-22) * p.t2 * 0.5 + 0x1.0518752509928p-34 * p.t3 * (1.0 / 3.0) + (-0x1.03e94c0ab008ap-48) * p.t4 * 0.25 + (p.rb ? (-0x1.19f4860ca78bdp+1) : (-0x1.e701974f118b1p+4))) : (-0x1.3e9e76d5cfaadp+15 * p.tm2 * 0.5 - (-0x1.907594d0dcfccp+9) * p.tm1 + 0x1.06ded6bfeabc2p+3 * p.lnT + (-0x1.a00f5e57224a9p-7) * p.T + 0x1.2634c3b74493ep-16 * p.t2 * 0.5 + (-0x1.9d4cb55199da9p-27) * p.t3 * (1.0 / 3.0) + 0x1.da045b502c793p-39 * p.t4 * 0.25 + (-0x1.e701974f118b1p+4));
}
template <> __device__ __forceinline__ double cp_r_spec<5>(const TPow &p)
{
    return p.hi ? (0x1.11d599a1cac08p+19 * p.tm2 + (-0x1.a29342bb66730p+9) * p.tm1 + 0x1.7cd8beb74f25fp+1 + 0x1.48450422d75b8p-10 * p.T + (-0x1.91a8060fc0cc0p-22) * p.t2 + 0x1.0518752509928p-34 * p.t3 + (-0x1.03e94c0ab008ap-48) * p.t4) : (0x1.3e9e76d5cfaadp+15 * p.tm2 + (-0x1.907594d0dcfccp+9) * p.tm1 + 0x1.06ded6bfeabc2p+3 + (-0x1.a00f5e57224a9p-7) * p.T + 0x1.2634c3b74493ep-16 * p.t2 + (-0x1.9d4cb55199da9p-27) * p.t3 + 0x1.da045b502c793p-39 * p.t4);
}
template <> __device__ __forceinline__ double h_r_spec<6>(const TPow &p)
{
    return p.hi ? (-0x1.6ba1406e978d5p+20 * p.tm1 + (-0x1.432d2602c9082p+12) * p.lnT + 0x1.69068d17ab177p+3 * p.T + (-0x1.515296b6985f4p-14) * p.t2 * 0.5 + (-0x1.38655d2945373p-26) * p.t3 * (1.0 / 3.0) + 0x1.e8decf9673d0bp-38 * p.t4 * 0.25 + (-0x1.164e393d55d7bp-51) * p.t5 * 0.2 + (p.rb ? 0x1.bb3415421c044p+13 : (-0x1.85b0306a2b170p+14))) : (-(-0x1.6a7b55f6fd220p+16) * p.tm1 + 0x1.872fe58a32f45p+10 * p.lnT + (-0x1.7e7e52abc9720p+2) * p.T + 0x1.0bf07bef07e1dp-5 * p.t2 * 0.5 + (-0x1.49db350f66c83p-15) * p.t3 * (1.0 / 3.0) + 0x1.af16365a726fdp-26 * p.t4 * 0.25 + (-0x1.c6efe6f8eebcbp-38) * p.t5 * 0.2 + (-0x1.85b0306a2b170p+14));
}
template <> __device__ __forceinline__ double s_r_spec<6>(const TPow &p)
{
    return p.hi ? (-0x1.6ba1406e978d5p+20 * p.tm2 * 0.5 - (-0x1.432d2602c9082p+12) * p.tm1 + 0x1.69068d17ab177p+3 * p.lnT + (-0x1.515296b6985f4p-14) * p.T + (-0x1.38655d2945373p-26) * p.t2 * 0.5 + 0x1.e8decf9673d0bp-38 * p.t3 * (1.0 / 3.0) + (-0x1.164e393d55d7bp-51) * p.t4 * 0.25 + (p.rb ? (-0x1.7411861f6951dp+5) : 0x1.d62c86f6ffa64p+5)) : (-(-0x1.6a7b55f6fd220p+16) * p.tm2 * 0.5 - 0x1.872fe58a32f45p+10 * p.tm1 + (-0x1.7e7e52abc9720p+2) * p.lnT + 0x1.0bf07bef07e1dp-5 * p.T + (-0x1.49db350f66c83p-15) * p.t2 * 0.5 + 0x1.af16365a726fdp-26 * p.t3 * (1.0 / 3.0) + (-0x1.c6efe6f8eebcbp-38) * p.t4 * 0.25 + 0x1.d62c86f6ffa64p+5);
}
template <> __device__ __forceinline__ double cp_r_spec<6>(const TPow &p)
{
    return p.hi ? (0x1.6ba1406e978d5p+20 * p.tm2 + (-0x1.432d2602c9082p+12) * p.tm1 + 0x1.69068d17ab177p+3 + (-0x1.515296b6985f4p-14) * p.T + (-0x1.38655d2945373p-26) * p.t2 + 0x1.e8decf9673d0bp-38 * p.t3 + (-0x1.164e393d55d7bp-51) * p.t4) : ((-0x1.6a7b55f6fd220p+16) * p.tm2 + 0x1.872fe58a32f45p+10 * p.tm1 + (-0x1.7e7e52abc9720p+2) + 0x1.0bf07bef07e1dp-5 * p.T + (-0x1.49db350f66c83p-15) * p.t2 + 0x1.af16365a726fdp-26 * p.t3 + (-0x1.c6efe6f8eebcbp-38) * p.t4);
}
template <> __device__ __forceinline__ double h_r_spec<7>(const TPow &p)
{
    return p.hi ? (-(-0x1.ba0edb9581062p+20) * p.tm1 + 0x1.3633128e0c9dap+12 * p.lnT + (-0x1.0a1c9b1edd6e6p+0) * p.T + 0x1.2ada98cd1ee1dp-8 * p.t2 * 0.5 + (-0x1.1d0a6cf1d43c0p-20) * p.t3 * (1.0 / 3.0) + 0x1.f762e3002e92cp-34 * p.t4 * 0.25 + (-0x1.5737068b814bfp-48) * p.t5 * 0.2 + (p.rb ? (-0x1.f420b0068db8cp+14) : (-0x1.6f159d883ba34p+12))) : (-(-0x1.28d4d34d6a162p+16) * p.tm1 + 0x1.4c58921ccd962p+10 * p.lnT + (-0x1.2b5a54345fae1p+2) * p.T + 0x1.9af6123d5cbe6p-6 * p.t2 * 0.5 + (-0x1.f86a684e1dea7p-16) * p.t3 * (1.0 / 3.0) + 0x1.45a95f43bda8ep-26 * p.t4 * 0.25 + (-0x1.53c7bcb8b40e2p-38) * p.t5 * 0.2 + (-0x1.6f159d883ba34p+12));
}
template <> __device__ __forceinline__ double s_r_spec<7>(const TPow &p)
{
    return p.hi ? (-(-0x1.ba0edb9581062p+20) * p.tm2 * 0.5 - 0x1.3633128e0c9dap+12 * p.tm1 + (-0x1.0a1c9b1edd6e6p+0) * p.lnT + 0x1.2ada98cd1ee1dp-8 * p.T + (-0x1.1d0a6cf1d43c0p-20) * p.t2 * 0.5 + 0x1.f762e3002e92cp-34 * p.t3 * (1.0 / 3.0) + (-0x1.5737068b814bfp-48) * p.t4 * 0.25 + (p.rb ? 0x1.45591b59f899ep+5 : 0x1.9f7cf8c9aad96p+5)) : (-(-0x1.28d4d34d6a162p+16) * p.tm2 * 0.5 - 0x1.4c58921ccd962p+10 * p.tm1 + (-0x1.2b5a54345fae1p+2) * p.lnT + 0x1.9af6123d5cbe6p-6 * p.T + (-0x1.f86a684e1dea7p-16) * p.t2 * 0.5 + 0x1.45a95f43bda8ep-26 * p.t3 * (1.0 / 3.0) + (-0x1.53c7bcb8b40e2p-38) * p.t4 * 0.25 + 0x1.9f7cf8c9aad96p+5);
}
template <> __device__ __forceinline__ double cp_r_spec<7>(const TPow &p)
{
    return p.hi ? ((-0x1.ba0edb9581062p+20) * p.tm2 + 0x1.3633128e0c9dap+12 * p.tm1 + (-0x1.0a1c9b1edd6e6p+0) + 0x1.2ada98cd1ee1dp-8 * p.T + (-0x1.1d0a6cf1d43c0p-20) * p.t2 + 0x1.f762e3002e92cp-34 * p.t3 + (-0x1.5737068b814bfp-48) * p.t4) : ((-0x1.28d4d34d6a162p+16) * p.tm2 + 0x1.4c58921ccd962p+10 * p.tm1 + (-0x1.2b5a54345fae1p+2) + 0x1.9af6123d5cbe6p-6 * p.T + (-0x1.f86a684e1dea7p-16) * p.t2 + 0x1.45a95f43bda8ep-26 * p.t3 + (-0x1.53c7bcb8b40e2p-38) * p.t4);
}
template <> __device__ __forceinline__ double h_r_spec<8>(const TPow &p)
{
    return p.hi ? (-0x1.1ef80cfdf3b64p+19 * p.tm1 + (-0x1.17e7f867f0aa2p+11) * p.lnT + 0x1.8448e56199222p+2 * p.T + (-0x1.41e576be829a1p-11) * p.t2 * 0.5 + 0x1.405cf082ec2ddp-23 * p.t3 * (1.0 / 3.0) + (-0x1.5250f8b15de24p-36) * p.t4 * 0.25 + 0x1.32166731f41f3p-50 * p.t5 * 0.2 + (p.rb ? 0x1.9100d54c985f0p+13 : 0x1.636c4c8bc9cd4p+9)) : (-0x1.595edc21187e8p+14 * p.tm1 + (-0x1.7dd89f623076cp+8) * p.lnT + 0x1.854b95d594c77p+2 * p.T + (-0x1.178a7f32adaccp-7) * p.t2 * 0.5 + 0x1.d09c33b406855p-17 * p.t3 * (1.0 / 3.0) + (-0x1.4abd6047b3e3cp-27) * p.t4 * 0.25 + 0x1.629df8198e88ap-39 * p.t5 * 0.2 + 0x1.636c4c8bc9cd4p+9);
}
template <> __device__ __forceinline__ double s_r_spec<8>(const TPow &p)
{
    return p.hi ? (-0x1.1ef80cfdf3b64p+19 * p.tm2 * 0.5 - (-0x1.17e7f867f0aa2p+11) * p.tm1 + 0x1.8448e56199222p+2 * p.lnT + (-0x1.41e576be829a1p-11) * p.T + 0x1.405cf082ec2ddp-23 * p.t2 * 0.5 + (-0x1.5250f8b15de24p-36) * p.t3 * (1.0 / 3.0) + 0x1.32166731f41f3p-50 * p.t4 * 0.25 + (p.rb ? (-0x1.fbb98d0f1ca88p+3) : (-0x1.58523a0991235p+3))) : (-0x1.595edc21187e8p+14 * p.tm2 * 0.5 - (-0x1.7dd89f623076cp+8) * p.tm1 + 0x1.854b95d594c77p+2 * p.lnT + (-0x1.178a7f32adaccp-7) * p.T + 0x1.d09c33b406855p-17 * p.t2 * 0.5 + (-0x1.4abd6047b3e3cp-27) * p.t3 * (1.0 / 3.0) + 0x1.629df8198e88ap-39 * p.t4 * 0.25 + (-0x1.58523a0991235p+3));
}
template <> __device__ __forceinline__ double cp_r_spec<8>(const TPow &p)
{
    return p.hi ? (0x1.1ef80cfdf3b64p+19 * p.tm2 + (-0x1.17e7f867f0aa2p+11) * p.tm1 + 0x1.8448e56199222p+2 + (-0x1.41e576be829a1p-11) * p.T + 0x1.405cf082ec2ddp-23 * p.t2 + (-0x1.5250f8b15de24p-36) * p.t3 + 0x1.32166731f41f3p-50 * p.t4) : (0x1.595edc21187e8p+14 * p.tm2 + (-0x1.7dd89f623076cp+8) * p.tm1 + 0x1.854b95d594c77p+2 + (-0x1.178a7f32adaccp-7) * p.T + 0x1.d09c33b406855p-17 * p.t2 + (-0x1.4abd6047b3e3cp-27) * p.t3 + 0x1.629df8198e88ap-39 * p.t4);
}

// Gibbs energies G_s = R (H_s/R - T S_s/R) in J/mol
__device__ __forceinline__ void gibbs_spec(const TPow &p, double G[NS])
{
    G[0] = R_GAS * h_r_spec<0>(p) - (R_GAS * s_r_spec<0>(p)) * p.T;
    G[1] = R_GAS * h_r_spec<1>(p) - (R_GAS * s_r_spec<1>(p)) * p.T;
    G[2] = R_GAS * h_r_spec<2>(p) - (R_GAS * s_r_spec<2>(p)) * p.T;
    G[3] = R_GAS * h_r_spec<3>(p) - (R_GAS * s_r_spec<3>(p)) * p.T;
    G[4] = R_GAS * h_r_spec<4>(p) - (R_GAS * s_r_spec<4>(p)) * p.T;
    G[5] = R_GAS * h_r_spec<5>(p) - (R_GAS * s_r_spec<5>(p)) * p.T;
    G[6] = R_GAS * h_r_spec<6>(p) - (R_GAS * s_r_spec<6>(p)) * p.T;
    G[7] = R_GAS * h_r_spec<7>(p) - (R_GAS * s_r_spec<7>(p)) * p.T;
    G[8] = R_GAS * h_r_spec<8>(p) - (R_GAS * s_r_spec<8>(p)) * p.T;
}

// H/R, S/R and Cp/R of every species at one temperature
__device__ __forceinline__ void thermo_spec(const TPow &p, double h[NS], double sr[NS], double cp[NS])
{
    h[0] = h_r_spec<0>(p);
    sr[0] = s_r_spec<0>(p);
    cp[0] = cp_r_spec<0>(p);
    h[1] = h_r_spec<1>(p);
    sr[1] = s_r_spec<1>(p);
    cp[1] = cp_r_spec<1>(p);
    h[2] = h_r_spec<2>(p);
    sr[2] = s_r_spec<2>(p);
    cp[2] = cp_r_spec<2>(p);
    h[3] = h_r_spec<3>(p);
    sr[3] = s_r_spec<3>(p);
    cp[3] = cp_r_spec<3>(p);
    h[4] = h_r_spec<4>(p);
    sr[4] = s_r_spec<4>(p);
    cp[4] = cp_r_spec<4>(p);
    h[5] = h_r_spec<5>(p);
    sr[5] = s_r_spec<5>(p);
    cp[5] = cp_r_spec<5>(p);
    h[6] = h_r_spec<6>(p);
    sr[6] = s_r_spec<6>(p);
    cp[6] = cp_r_spec<6>(p);
    h[7] = h_r_spec<7>(p);
    sr[7] = s_r_spec<7>(p);
    cp[7] = cp_r_spec<7>(p);
    h[8] = h_r_spec<8>(p);
    sr[8] = s_r_spec<8>(p);
    cp[8] = cp_r_spec<8>(p);
}

// Reaction::Diagonalized per cell: CMS (kg/m^3/s) and MD(s, s)
__device__ __forceinline__ void diagonalized_spec(const TPow &p, const double G[NS], const double Mc[NS],
                                                  const double Di[NS], const double PT[NS], double CMS[NS],
                                                  double MD[NS])
{
    double Wi[NS];
    // 1/Di, with a subnormal Di (and its numerator) scaled by 2^64 so that the
    // reciprocal stays finite; the scalings are exact
    double iDi[NS], sDi[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        sDi[s] = fabs(Di[s]) < 0x1p-1022 ? 0x1p+64 : 1.0;
        iDi[s] = Di[s] == 0.0 ? 0.0 : 1.0 / (Di[s] * sDi[s]);
    }
    const double tdep = 1.0 / (RU_CAL * (p.T * p.T));
#pragma unroll
    for (int s = 0; s < NS; s++) { Wi[s] = 0.0; MD[s] = 0.0; }
    {
        // reaction 1
        const double kf = 0x1.6bcc41e900000p+46 * 1.0 * exp(-0x1.b5be07fcb923ap+15 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[0] + (-0x1.0000000000000p+0) * G[4] + (-0x1.0000000000000p+0) * G[5] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[4] * Mc[5];
        const double rb = Mc[0] * Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.b5be07fcb923ap+15 * tdep);
        Wi[0] += 0x1.0000000000000p+0 * tb * rr;
        MD[0] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb);
        Wi[4] += (-0x1.0000000000000p+0) * tb * rr;
        MD[4] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[4]) * iDi[4] + wjh2 * PT[4]) * tb);
        Wi[5] += (-0x1.0000000000000p+0) * tb * rr;
        MD[5] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[5]) * iDi[5] + wjh2 * PT[5]) * tb);
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        MD[7] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 2
        const double kf = 0x1.d8efef4880000p+47 * 1.0 * exp(-0x1.06a537e90ff97p+14 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+0 * G[1] + 0x1.0000000000000p+0 * G[3] + (-0x1.0000000000000p+0) * G[4];
        const double rf = Mc[0] * Mc[4];
        const double rb = Mc[1] * Mc[3];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.06a537e90ff97p+14 * tdep);
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        MD[0] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb);
        Wi[1] += 0x1.0000000000000p+0 * tb * rr;
        MD[1] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[1]) * iDi[1] + wjh2 * PT[1]) * tb);
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        MD[3] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
        Wi[4] += (-0x1.0000000000000p+0) * tb * rr;
        MD[4] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[4]) * iDi[4] + wjh2 * PT[4]) * tb);
    }
    {
        // reaction 3
        const double kf = 0x1.0c388d0000000p+34 * p.T * exp(-0x1.1647837b4a234p+13 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[0] + (-0x1.0000000000000p+0) * G[1] + 0x1.0000000000000p+0 * G[3] + (-0x1.0000000000000p+0) * G[5];
        const double rf = Mc[1] * Mc[5];
        const double rb = Mc[0] * Mc[3];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.0000000000000p+0 * p.tm1 + 0x1.1647837b4a234p+13 * tdep);
        Wi[0] += 0x1.0000000000000p+0 * tb * rr;
        MD[0] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb);
        Wi[1] += (-0x1.0000000000000p+0) * tb * rr;
        MD[1] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[1]) * iDi[1] + wjh2 * PT[1]) * tb);
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        MD[3] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
        Wi[5] += (-0x1.0000000000000p+0) * tb * rr;
        MD[5] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[5]) * iDi[5] + wjh2 * PT[5]) * tb);
    }
    {
        // reaction 4
        const double kf = 0x1.402462f600000p+44 * 1.0 * exp(-0x1.420d8e8a71de7p+12 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[0] + 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[3] + (-0x1.0000000000000p+0) * G[5];
        const double rf = Mc[3] * Mc[5];
        const double rb = Mc[0] * Mc[2];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.420d8e8a71de7p+12 * tdep);
        Wi[0] += 0x1.0000000000000p+0 * tb * rr;
        MD[0] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb);
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        MD[2] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[2]) * iDi[2] + wjh2 * PT[2]) * tb);
        Wi[3] += (-0x1.0000000000000p+0) * tb * rr;
        MD[3] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
        Wi[5] += (-0x1.0000000000000p+0) * tb * rr;
        MD[5] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[5]) * iDi[5] + wjh2 * PT[5]) * tb);
    }
    {
        // reaction 5
        const double kf = 0x1.6eb550c600000p+42 * 1.0 * exp(-0x1.10a6b1c432ca5p+10 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[1] + 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+1) * G[3];
        const double rf = (Mc[3] * Mc[3]);
        const double rb = Mc[1] * Mc[2];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.10a6b1c432ca5p+10 * tdep);
        Wi[1] += 0x1.0000000000000p+0 * tb * rr;
        MD[1] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[1]) * iDi[1] + wjh2 * PT[1]) * tb);
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        MD[2] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[2]) * iDi[2] + wjh2 * PT[2]) * tb);
        Wi[3] += (-0x1.0000000000000p+1) * tb * rr;
        MD[3] += (-0x1.0000000000000p+1) * ((((kf * 0x1.0000000000000p+1 * rf) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
    }
    {
        // reaction 6
        const double kf = 0x1.2a27d53bc0487p+74 * p.tm2;
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[3];
        const double rf = Mc[0] * Mc[3];
        const double rb = Mc[2];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.8000000000000p+2 + Mc[3] + Mc[4] + Mc[5] + Mc[6] + Mc[7] + Mc[8];
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * ((-0x1.0000000000000p+1) * p.tm1);
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        MD[0] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb + rr * 0x1.fbf77c89c7e90p-1);
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        MD[2] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[2]) * iDi[2] + wjh2 * PT[2]) * tb + rr * 0x1.550b381dd224bp-2);
        Wi[3] += (-0x1.0000000000000p+0) * tb * rr;
        MD[3] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb + rr * 0x1.e1aca45c4cb5ep-5);
    }
    {
        // reaction 7
        const double kf = 0x1.1c37937e08000p+59 * p.tm1;
        const double dg = (-0x1.0000000000000p+1) * G[0] + 0x1.0000000000000p+0 * G[5];
        const double rf = (Mc[0] * Mc[0]);
        const double rb = Mc[5];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.8000000000000p+2 + Mc[3] + Mc[4] + Mc[5] * 0x1.0000000000000p+1 + Mc[6] + Mc[7] + Mc[8];
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * ((-0x1.0000000000000p+0) * p.tm1);
        Wi[0] += (-0x1.0000000000000p+1) * tb * rr;
        MD[0] += (-0x1.0000000000000p+1) * ((((kf * 0x1.0000000000000p+1 * rf) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb + rr * 0x1.fbf77c89c7e90p-1);
        Wi[5] += 0x1.0000000000000p+0 * tb * rr;
        MD[5] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[5]) * iDi[5] + wjh2 * PT[5]) * tb + rr * 0x1.fbf77c89c7e90p-1);
    }
    {
        // reaction 8
        const double kf = 0x1.aa535d3d0c000p+55 * exp((-0x1.3333333333333p-1) * p.lnT);
        const double dg = (-0x1.0000000000000p+0) * G[0] + (-0x1.0000000000000p+0) * G[1] + 0x1.0000000000000p+0 * G[3];
        const double rf = Mc[0] * Mc[1];
        const double rb = Mc[3];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.4000000000000p+2 + Mc[3] + Mc[4] + Mc[5] + Mc[6] + Mc[7] + Mc[8];
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * ((-0x1.3333333333333p-1) * p.tm1);
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        MD[0] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb + rr * 0x1.fbf77c89c7e90p-1);
        Wi[1] += (-0x1.0000000000000p+0) * tb * rr;
        MD[1] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[1]) * iDi[1] + wjh2 * PT[1]) * tb + rr * 0x1.0002752b5049bp-4);
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        MD[3] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb + rr * 0x1.e1aca45c4cb5ep-5);
    }
    {
        // reaction 9
        const double kf = 0x1.dd7c1681d0000p+50 * 1.0 * exp(-(-0x1.f446e2eb1c433p+9) / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + (-0x1.0000000000000p+0) * G[4] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[0] * Mc[4];
        const double rb = Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.0000000000000p+4 + Mc[3] + Mc[4] + Mc[5] * 0x1.0000000000000p+1 + Mc[6] + Mc[7] + Mc[8];
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * ((-0x1.f446e2eb1c433p+9) * tdep);
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        MD[0] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb + rr * 0x1.fbf77c89c7e90p-1);
        Wi[4] += (-0x1.0000000000000p+0) * tb * rr;
        MD[4] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[4]) * iDi[4] + wjh2 * PT[4]) * tb + rr * 0x1.0002752b5049bp-5);
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        MD[7] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb + rr * 0x1.f0622ad29be6cp-6);
    }
    {
        // reaction 10
        const double kf = 0x1.b48eb57e00000p+45 * 1.0 * exp(-(-0x1.c23fcd35a8588p+10) / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+1) * G[1] + 0x1.0000000000000p+0 * G[4];
        const double rf = (Mc[1] * Mc[1]);
        const double rb = Mc[4];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] + Mc[3] + Mc[4] + Mc[5] + Mc[6] + Mc[7] + Mc[8];
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * ((-0x1.c23fcd35a8588p+10) * tdep);
        Wi[1] += (-0x1.0000000000000p+1) * tb * rr;
        MD[1] += (-0x1.0000000000000p+1) * ((((kf * 0x1.0000000000000p+1 * rf) * sDi[1]) * iDi[1] + wjh2 * PT[1]) * tb + rr * 0x1.0002752b5049bp-4);
        Wi[4] += 0x1.0000000000000p+0 * tb * rr;
        MD[4] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[4]) * iDi[4] + wjh2 * PT[4]) * tb + rr * 0x1.0002752b5049bp-5);
    }
    {
        // reaction 11
        const double kf = 0x1.fd51291300000p+46 * 1.0 * exp(-0x1.0e25c5d638866p+10 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+1 * G[3] + (-0x1.0000000000000p+0) * G[7];
        const double rf = Mc[0] * Mc[7];
        const double rb = (Mc[3] * Mc[3]);
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.0e25c5d638866p+10 * tdep);
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        MD[0] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb);
        Wi[3] += 0x1.0000000000000p+1 * tb * rr;
        MD[3] += 0x1.0000000000000p+1 * ((((-kb * 0x1.0000000000000p+1 * rb) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
        Wi[7] += (-0x1.0000000000000p+0) * tb * rr;
        MD[7] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 12
        const double kf = 0x1.2309ce5400000p+43 * 1.0 * exp(-0x1.0e25c5d638866p+10 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+0 * G[1] + 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[7];
        const double rf = Mc[0] * Mc[7];
        const double rb = Mc[1] * Mc[2];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.0e25c5d638866p+10 * tdep);
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        MD[0] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb);
        Wi[1] += 0x1.0000000000000p+0 * tb * rr;
        MD[1] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[1]) * iDi[1] + wjh2 * PT[1]) * tb);
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        MD[2] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[2]) * iDi[2] + wjh2 * PT[2]) * tb);
        Wi[7] += (-0x1.0000000000000p+0) * tb * rr;
        MD[7] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 13
        const double kf = 0x1.b48eb57e00000p+43 * 1.0 * exp(-0x1.db42b367a0f91p+9 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[1] + 0x1.0000000000000p+0 * G[3] + 0x1.0000000000000p+0 * G[4] + (-0x1.0000000000000p+0) * G[7];
        const double rf = Mc[1] * Mc[7];
        const double rb = Mc[3] * Mc[4];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.db42b367a0f91p+9 * tdep);
        Wi[1] += (-0x1.0000000000000p+0) * tb * rr;
        MD[1] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[1]) * iDi[1] + wjh2 * PT[1]) * tb);
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        MD[3] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
        Wi[4] += 0x1.0000000000000p+0 * tb * rr;
        MD[4] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[4]) * iDi[4] + wjh2 * PT[4]) * tb);
        Wi[7] += (-0x1.0000000000000p+0) * tb * rr;
        MD[7] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 14
        const double kf = 0x1.d1a94a2000000p+42 * 1.0;
        const double dg = 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[3] + 0x1.0000000000000p+0 * G[4] + (-0x1.0000000000000p+0) * G[7];
        const double rf = Mc[3] * Mc[7];
        const double rb = Mc[2] * Mc[4];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0.0);
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        MD[2] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[2]) * iDi[2] + wjh2 * PT[2]) * tb);
        Wi[3] += (-0x1.0000000000000p+0) * tb * rr;
        MD[3] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
        Wi[4] += 0x1.0000000000000p+0 * tb * rr;
        MD[4] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[4]) * iDi[4] + wjh2 * PT[4]) * tb);
        Wi[7] += (-0x1.0000000000000p+0) * tb * rr;
        MD[7] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 15
        const double kf = 0x1.d1a94a2000000p+40 * 1.0;
        const double dg = 0x1.0000000000000p+0 * G[4] + 0x1.0000000000000p+0 * G[6] + (-0x1.0000000000000p+1) * G[7];
        const double rf = (Mc[7] * Mc[7]);
        const double rb = Mc[4] * Mc[6];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0.0);
        Wi[4] += 0x1.0000000000000p+0 * tb * rr;
        MD[4] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[4]) * iDi[4] + wjh2 * PT[4]) * tb);
        Wi[6] += 0x1.0000000000000p+0 * tb * rr;
        MD[6] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[6]) * iDi[6] + wjh2 * PT[6]) * tb);
        Wi[7] += (-0x1.0000000000000p+1) * tb * rr;
        MD[7] += (-0x1.0000000000000p+1) * ((((kf * 0x1.0000000000000p+1 * rf) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 16
        const double kf = 0x1.45f680b000000p+40 * 1.0 * exp(-0x1.c23fcd35a8588p+11 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+0 * G[5] + (-0x1.0000000000000p+0) * G[6] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[0] * Mc[6];
        const double rb = Mc[5] * Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.c23fcd35a8588p+11 * tdep);
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        MD[0] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[0]) * iDi[0] + wjh2 * PT[0]) * tb);
        Wi[5] += 0x1.0000000000000p+0 * tb * rr;
        MD[5] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[5]) * iDi[5] + wjh2 * PT[5]) * tb);
        Wi[6] += (-0x1.0000000000000p+0) * tb * rr;
        MD[6] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[6]) * iDi[6] + wjh2 * PT[6]) * tb);
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        MD[7] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 17
        const double kf = 0x1.977420dc00000p+43 * 1.0 * exp(-0x1.9038b6ae7d567p+12 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[1] + 0x1.0000000000000p+0 * G[3] + (-0x1.0000000000000p+0) * G[6] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[1] * Mc[6];
        const double rb = Mc[3] * Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.9038b6ae7d567p+12 * tdep);
        Wi[1] += (-0x1.0000000000000p+0) * tb * rr;
        MD[1] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[1]) * iDi[1] + wjh2 * PT[1]) * tb);
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        MD[3] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
        Wi[6] += (-0x1.0000000000000p+0) * tb * rr;
        MD[6] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[6]) * iDi[6] + wjh2 * PT[6]) * tb);
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        MD[7] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 18
        const double kf = 0x1.6311155200000p+42 * 1.0 * exp(-0x1.65b3212d77319p+10 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[3] + (-0x1.0000000000000p+0) * G[6] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[3] * Mc[6];
        const double rb = Mc[2] * Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.65b3212d77319p+10 * tdep);
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        MD[2] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[2]) * iDi[2] + wjh2 * PT[2]) * tb);
        Wi[3] += (-0x1.0000000000000p+0) * tb * rr;
        MD[3] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb);
        Wi[6] += (-0x1.0000000000000p+0) * tb * rr;
        MD[6] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[6]) * iDi[6] + wjh2 * PT[6]) * tb);
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        MD[7] += 0x1.0000000000000p+0 * ((((-kb * 0x1.0000000000000p+0 * rb) * sDi[7]) * iDi[7] + wjh2 * PT[7]) * tb);
    }
    {
        // reaction 19
        const double kf = 0x1.aa535d3d0c000p+56 * 1.0 * exp(-0x1.63aa6b923a29cp+15 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+1 * G[3] + (-0x1.0000000000000p+0) * G[6];
        const double rf = Mc[6];
        const double rb = (Mc[3] * Mc[3]);
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.9f06f69446738p-4;
        const double kb = kf / (kp * (1.0 / (R_GAS * p.T)));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.e000000000000p+3 + Mc[3] + Mc[4] + Mc[5] + Mc[6] + Mc[7] + Mc[8];
        if (tb == 0.0) tb = 1.0;
        const double rr = kf * rf - kb * rb;
        const double wjh2 = rr * (0x1.63aa6b923a29cp+15 * tdep);
        Wi[3] += 0x1.0000000000000p+1 * tb * rr;
        MD[3] += 0x1.0000000000000p+1 * ((((-kb * 0x1.0000000000000p+1 * rb) * sDi[3]) * iDi[3] + wjh2 * PT[3]) * tb + rr * 0x1.e1aca45c4cb5ep-5);
        Wi[6] += (-0x1.0000000000000p+0) * tb * rr;
        MD[6] += (-0x1.0000000000000p+0) * ((((kf * 0x1.0000000000000p+0 * rf) * sDi[6]) * iDi[6] + wjh2 * PT[6]) * tb + rr * 0x1.e1aca45c4cb5ep-6);
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        CMS[s] = (cM.mw[s] * Wi[s]) * 1e3;
        MD[s] = cM.mw[s] * MD[s];
    }
}

// Point-implicit trapezoid production/loss (src/Reaction.cpp:455-482);
// rtb_mode 0: R_TB -> 1 when 0, 1: left as summed, 2: forced to 0
__device__ __forceinline__ void trap_rates_spec(const TPow &p, const double Mc[NS], int rtb_mode, double Wi[NS],
                                                double Pv[NS], double Qv[NS])
{
    double G[NS];
    gibbs_spec(p, G);
#pragma unroll
    for (int s = 0; s < NS; s++) { Wi[s] = 0.0; Pv[s] = 0.0; Qv[s] = 0.0; }
    {
        // reaction 1
        const double kf = 0x1.6bcc41e900000p+46 * 1.0 * exp(-0x1.b5be07fcb923ap+15 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[0] + (-0x1.0000000000000p+0) * G[4] + (-0x1.0000000000000p+0) * G[5] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[4] * Mc[5];
        const double rb = Mc[0] * Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += 0x1.0000000000000p+0 * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kf * rf;
        Pv[0] += 0x1.0000000000000p+0 * kb * rb;
        Wi[4] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[4] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[4] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[5] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[5] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[5] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kf * rf;
        Pv[7] += 0x1.0000000000000p+0 * kb * rb;
    }
    {
        // reaction 2
        const double kf = 0x1.d8efef4880000p+47 * 1.0 * exp(-0x1.06a537e90ff97p+14 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+0 * G[1] + 0x1.0000000000000p+0 * G[3] + (-0x1.0000000000000p+0) * G[4];
        const double rf = Mc[0] * Mc[4];
        const double rb = Mc[1] * Mc[3];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[0] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[1] += 0x1.0000000000000p+0 * tb * rr;
        Qv[1] += 0x1.0000000000000p+0 * kf * rf;
        Pv[1] += 0x1.0000000000000p+0 * kb * rb;
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kf * rf;
        Pv[3] += 0x1.0000000000000p+0 * kb * rb;
        Wi[4] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[4] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[4] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
    {
        // reaction 3
        const double kf = 0x1.0c388d0000000p+34 * p.T * exp(-0x1.1647837b4a234p+13 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[0] + (-0x1.0000000000000p+0) * G[1] + 0x1.0000000000000p+0 * G[3] + (-0x1.0000000000000p+0) * G[5];
        const double rf = Mc[1] * Mc[5];
        const double rb = Mc[0] * Mc[3];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += 0x1.0000000000000p+0 * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kf * rf;
        Pv[0] += 0x1.0000000000000p+0 * kb * rb;
        Wi[1] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[1] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[1] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kf * rf;
        Pv[3] += 0x1.0000000000000p+0 * kb * rb;
        Wi[5] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[5] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[5] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
    {
        // reaction 4
        const double kf = 0x1.402462f600000p+44 * 1.0 * exp(-0x1.420d8e8a71de7p+12 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[0] + 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[3] + (-0x1.0000000000000p+0) * G[5];
        const double rf = Mc[3] * Mc[5];
        const double rb = Mc[0] * Mc[2];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += 0x1.0000000000000p+0 * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kf * rf;
        Pv[0] += 0x1.0000000000000p+0 * kb * rb;
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        Qv[2] += 0x1.0000000000000p+0 * kf * rf;
        Pv[2] += 0x1.0000000000000p+0 * kb * rb;
        Wi[3] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[3] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[5] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[5] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[5] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
    {
        // reaction 5
        const double kf = 0x1.6eb550c600000p+42 * 1.0 * exp(-0x1.10a6b1c432ca5p+10 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[1] + 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+1) * G[3];
        const double rf = (Mc[3] * Mc[3]);
        const double rb = Mc[1] * Mc[2];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[1] += 0x1.0000000000000p+0 * tb * rr;
        Qv[1] += 0x1.0000000000000p+0 * kf * rf;
        Pv[1] += 0x1.0000000000000p+0 * kb * rb;
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        Qv[2] += 0x1.0000000000000p+0 * kf * rf;
        Pv[2] += 0x1.0000000000000p+0 * kb * rb;
        Wi[3] += (-0x1.0000000000000p+1) * tb * rr;
        Qv[3] += 0x1.0000000000000p+1 * kb * rb * tb;
        Pv[3] += 0x1.0000000000000p+1 * kf * rf * tb;
    }
    {
        // reaction 6
        const double kf = 0x1.2a27d53bc0487p+74 * p.tm2;
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[3];
        const double rf = Mc[0] * Mc[3];
        const double rb = Mc[2];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.8000000000000p+2 + Mc[3] + Mc[4] + Mc[5] + Mc[6] + Mc[7] + Mc[8];
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[0] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        Qv[2] += 0x1.0000000000000p+0 * kf * rf;
        Pv[2] += 0x1.0000000000000p+0 * kb * rb;
        Wi[3] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[3] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
    {
        // reaction 7
        const double kf = 0x1.1c37937e08000p+59 * p.tm1;
        const double dg = (-0x1.0000000000000p+1) * G[0] + 0x1.0000000000000p+0 * G[5];
        const double rf = (Mc[0] * Mc[0]);
        const double rb = Mc[5];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.8000000000000p+2 + Mc[3] + Mc[4] + Mc[5] * 0x1.0000000000000p+1 + Mc[6] + Mc[7] + Mc[8];
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += (-0x1.0000000000000p+1) * tb * rr;
        Qv[0] += 0x1.0000000000000p+1 * kb * rb * tb;
        Pv[0] += 0x1.0000000000000p+1 * kf * rf * tb;
        Wi[5] += 0x1.0000000000000p+0 * tb * rr;
        Qv[5] += 0x1.0000000000000p+0 * kf * rf;
        Pv[5] += 0x1.0000000000000p+0 * kb * rb;
    }
    {
        // reaction 8
        const double kf = 0x1.aa535d3d0c000p+55 * exp((-0x1.3333333333333p-1) * p.lnT);
        const double dg = (-0x1.0000000000000p+0) * G[0] + (-0x1.0000000000000p+0) * G[1] + 0x1.0000000000000p+0 * G[3];
        const double rf = Mc[0] * Mc[1];
        const double rb = Mc[3];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.4000000000000p+2 + Mc[3] + Mc[4] + Mc[5] + Mc[6] + Mc[7] + Mc[8];
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[0] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[1] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[1] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[1] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kf * rf;
        Pv[3] += 0x1.0000000000000p+0 * kb * rb;
    }
    {
        // reaction 9
        const double kf = 0x1.dd7c1681d0000p+50 * 1.0 * exp(-(-0x1.f446e2eb1c433p+9) / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + (-0x1.0000000000000p+0) * G[4] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[0] * Mc[4];
        const double rb = Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.0000000000000p+4 + Mc[3] + Mc[4] + Mc[5] * 0x1.0000000000000p+1 + Mc[6] + Mc[7] + Mc[8];
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[0] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[4] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[4] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[4] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kf * rf;
        Pv[7] += 0x1.0000000000000p+0 * kb * rb;
    }
    {
        // reaction 10
        const double kf = 0x1.b48eb57e00000p+45 * 1.0 * exp(-(-0x1.c23fcd35a8588p+10) / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+1) * G[1] + 0x1.0000000000000p+0 * G[4];
        const double rf = (Mc[1] * Mc[1]);
        const double rb = Mc[4];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.3bd0c106c229dp+3;
        const double kb = kf / (kp * (R_GAS * p.T));
        double tb = Mc[0] + Mc[1] + Mc[2] + Mc[3] + Mc[4] + Mc[5] + Mc[6] + Mc[7] + Mc[8];
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[1] += (-0x1.0000000000000p+1) * tb * rr;
        Qv[1] += 0x1.0000000000000p+1 * kb * rb * tb;
        Pv[1] += 0x1.0000000000000p+1 * kf * rf * tb;
        Wi[4] += 0x1.0000000000000p+0 * tb * rr;
        Qv[4] += 0x1.0000000000000p+0 * kf * rf;
        Pv[4] += 0x1.0000000000000p+0 * kb * rb;
    }
    {
        // reaction 11
        const double kf = 0x1.fd51291300000p+46 * 1.0 * exp(-0x1.0e25c5d638866p+10 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+1 * G[3] + (-0x1.0000000000000p+0) * G[7];
        const double rf = Mc[0] * Mc[7];
        const double rb = (Mc[3] * Mc[3]);
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[0] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[3] += 0x1.0000000000000p+1 * tb * rr;
        Qv[3] += 0x1.0000000000000p+1 * kf * rf;
        Pv[3] += 0x1.0000000000000p+1 * kb * rb;
        Wi[7] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[7] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
    {
        // reaction 12
        const double kf = 0x1.2309ce5400000p+43 * 1.0 * exp(-0x1.0e25c5d638866p+10 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+0 * G[1] + 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[7];
        const double rf = Mc[0] * Mc[7];
        const double rb = Mc[1] * Mc[2];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[0] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[1] += 0x1.0000000000000p+0 * tb * rr;
        Qv[1] += 0x1.0000000000000p+0 * kf * rf;
        Pv[1] += 0x1.0000000000000p+0 * kb * rb;
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        Qv[2] += 0x1.0000000000000p+0 * kf * rf;
        Pv[2] += 0x1.0000000000000p+0 * kb * rb;
        Wi[7] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[7] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
    {
        // reaction 13
        const double kf = 0x1.b48eb57e00000p+43 * 1.0 * exp(-0x1.db42b367a0f91p+9 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[1] + 0x1.0000000000000p+0 * G[3] + 0x1.0000000000000p+0 * G[4] + (-0x1.0000000000000p+0) * G[7];
        const double rf = Mc[1] * Mc[7];
        const double rb = Mc[3] * Mc[4];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[1] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[1] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[1] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kf * rf;
        Pv[3] += 0x1.0000000000000p+0 * kb * rb;
        Wi[4] += 0x1.0000000000000p+0 * tb * rr;
        Qv[4] += 0x1.0000000000000p+0 * kf * rf;
        Pv[4] += 0x1.0000000000000p+0 * kb * rb;
        Wi[7] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[7] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
    {
        // reaction 14
        const double kf = 0x1.d1a94a2000000p+42 * 1.0;
        const double dg = 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[3] + 0x1.0000000000000p+0 * G[4] + (-0x1.0000000000000p+0) * G[7];
        const double rf = Mc[3] * Mc[7];
        const double rb = Mc[2] * Mc[4];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        Qv[2] += 0x1.0000000000000p+0 * kf * rf;
        Pv[2] += 0x1.0000000000000p+0 * kb * rb;
        Wi[3] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[3] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[4] += 0x1.0000000000000p+0 * tb * rr;
        Qv[4] += 0x1.0000000000000p+0 * kf * rf;
        Pv[4] += 0x1.0000000000000p+0 * kb * rb;
        Wi[7] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[7] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
    {
        // reaction 15
        const double kf = 0x1.d1a94a2000000p+40 * 1.0;
        const double dg = 0x1.0000000000000p+0 * G[4] + 0x1.0000000000000p+0 * G[6] + (-0x1.0000000000000p+1) * G[7];
        const double rf = (Mc[7] * Mc[7]);
        const double rb = Mc[4] * Mc[6];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[4] += 0x1.0000000000000p+0 * tb * rr;
        Qv[4] += 0x1.0000000000000p+0 * kf * rf;
        Pv[4] += 0x1.0000000000000p+0 * kb * rb;
        Wi[6] += 0x1.0000000000000p+0 * tb * rr;
        Qv[6] += 0x1.0000000000000p+0 * kf * rf;
        Pv[6] += 0x1.0000000000000p+0 * kb * rb;
        Wi[7] += (-0x1.0000000000000p+1) * tb * rr;
        Qv[7] += 0x1.0000000000000p+1 * kb * rb * tb;
        Pv[7] += 0x1.0000000000000p+1 * kf * rf * tb;
    }
    {
        // reaction 16
        const double kf = 0x1.45f680b000000p+40 * 1.0 * exp(-0x1.c23fcd35a8588p+11 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[0] + 0x1.0000000000000p+0 * G[5] + (-0x1.0000000000000p+0) * G[6] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[0] * Mc[6];
        const double rb = Mc[5] * Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[0] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[0] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[0] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[5] += 0x1.0000000000000p+0 * tb * rr;
        Qv[5] += 0x1.0000000000000p+0 * kf * rf;
        Pv[5] += 0x1.0000000000000p+0 * kb * rb;
        Wi[6] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[6] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[6] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kf * rf;
        Pv[7] += 0x1.0000000000000p+0 * kb * rb;
    }
    {
        // reaction 17
        const double kf = 0x1.977420dc00000p+43 * 1.0 * exp(-0x1.9038b6ae7d567p+12 / (RU_CAL * p.T));
        const double dg = (-0x1.0000000000000p+0) * G[1] + 0x1.0000000000000p+0 * G[3] + (-0x1.0000000000000p+0) * G[6] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[1] * Mc[6];
        const double rb = Mc[3] * Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[1] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[1] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[1] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[3] += 0x1.0000000000000p+0 * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kf * rf;
        Pv[3] += 0x1.0000000000000p+0 * kb * rb;
        Wi[6] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[6] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[6] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kf * rf;
        Pv[7] += 0x1.0000000000000p+0 * kb * rb;
    }
    {
        // reaction 18
        const double kf = 0x1.6311155200000p+42 * 1.0 * exp(-0x1.65b3212d77319p+10 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+0 * G[2] + (-0x1.0000000000000p+0) * G[3] + (-0x1.0000000000000p+0) * G[6] + 0x1.0000000000000p+0 * G[7];
        const double rf = Mc[3] * Mc[6];
        const double rb = Mc[2] * Mc[7];
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.0000000000000p+0;
        const double kb = kf / (kp);
        double tb = 0.0;
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[2] += 0x1.0000000000000p+0 * tb * rr;
        Qv[2] += 0x1.0000000000000p+0 * kf * rf;
        Pv[2] += 0x1.0000000000000p+0 * kb * rb;
        Wi[3] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[3] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[3] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[6] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[6] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[6] += 0x1.0000000000000p+0 * kf * rf * tb;
        Wi[7] += 0x1.0000000000000p+0 * tb * rr;
        Qv[7] += 0x1.0000000000000p+0 * kf * rf;
        Pv[7] += 0x1.0000000000000p+0 * kb * rb;
    }
    {
        // reaction 19
        const double kf = 0x1.aa535d3d0c000p+56 * 1.0 * exp(-0x1.63aa6b923a29cp+15 / (RU_CAL * p.T));
        const double dg = 0x1.0000000000000p+1 * G[3] + (-0x1.0000000000000p+0) * G[6];
        const double rf = Mc[6];
        const double rb = (Mc[3] * Mc[3]);
        const double kp = exp(-dg / (R_GAS * p.T)) * 0x1.9f06f69446738p-4;
        const double kb = kf / (kp * (1.0 / (R_GAS * p.T)));
        double tb = Mc[0] + Mc[1] + Mc[2] * 0x1.e000000000000p+3 + Mc[3] + Mc[4] + Mc[5] + Mc[6] + Mc[7] + Mc[8];
        if (rtb_mode == 0) { if (tb == 0.0) tb = 1.0; } else if (rtb_mode == 2) { tb = 0.0; }
        const double rr = kf * rf - kb * rb;
        Wi[3] += 0x1.0000000000000p+1 * tb * rr;
        Qv[3] += 0x1.0000000000000p+1 * kf * rf;
        Pv[3] += 0x1.0000000000000p+1 * kb * rb;
        Wi[6] += (-0x1.0000000000000p+0) * tb * rr;
        Qv[6] += 0x1.0000000000000p+0 * kb * rb * tb;
        Pv[6] += 0x1.0000000000000p+0 * kf * rf * tb;
    }
#pragma unroll
    for (int s = 0; s < NS; s++) Wi[s] = cM.mw[s] * Wi[s];
}

}  // namespace h2ja919
}  // namespace eu3d
