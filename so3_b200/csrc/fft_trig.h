// Generated by gen_fft_trig.py: cos / sin (2 pi k / R), k = 0 .. (R-1)/2, for the odd
// radices of the DFT engine, at kTrigCos[TrigOff<R>::v + k].  Do not edit by hand.
// Indexed with compile-time offsets, the values are constant-bank operands.
#pragma once

namespace so3g {

template <int R>
struct TrigOff;
template <>
struct TrigOff<3> {
  static constexpr int v = 0;
};
template <>
struct TrigOff<5> {
  static constexpr int v = 2;
};
template <>
struct TrigOff<7> {
  static constexpr int v = 5;
};
template <>
struct TrigOff<11> {
  static constexpr int v = 9;
};
template <>
struct TrigOff<13> {
  static constexpr int v = 15;
};
template <>
struct TrigOff<17> {
  static constexpr int v = 22;
};
template <>
struct TrigOff<19> {
  static constexpr int v = 31;
};
template <>
struct TrigOff<23> {
  static constexpr int v = 41;
};
template <>
struct TrigOff<29> {
  static constexpr int v = 53;
};
template <>
struct TrigOff<31> {
  static constexpr int v = 68;
};
template <>
struct TrigOff<9> {
  static constexpr int v = 84;
};

static __constant__ double kTrigCos[89] = {
    0x1.0000000000000p+0, -0x1.0000000000000p-1, 0x1.0000000000000p+0, 0x1.3c6ef372fe950p-2,
    -0x1.9e3779b97f4a8p-1, 0x1.0000000000000p+0, 0x1.3f3a0e28bedd1p-1, -0x1.c7b90e3024582p-3,
    -0x1.cd4bca9cb5c71p-1, 0x1.0000000000000p+0, 0x1.aeb8c8764f0bap-1, 0x1.a9628d9c712b6p-2,
    -0x1.2375f640f44dbp-3, -0x1.4f49e7f775887p-1, -0x1.eb42a9bcd5057p-1, 0x1.0000000000000p+0,
    0x1.c55a7e00740e9p-1, 0x1.22d961ea71119p-1, 0x1.edb7debaa3ed8p-4, -0x1.6b1d8b2365da1p-2,
    -0x1.7f3ccd0032e0cp-1, -0x1.f11f493053d00p-1, 0x1.0000000000000p+0, 0x1.dd6d000370991p-1,
    0x1.7a5f6075d4884p-1, 0x1.c86fa2b2883cdp-2, 0x1.79ee63259b75ep-4, -0x1.183b1c61f0d01p-2,
    -0x1.348c86ed5f1bbp-1, -0x1.b34fa910ea3b9p-1, -0x1.f7484007faef3p-1, 0x1.0000000000000p+0,
    0x1.e442285231be1p-1, 0x1.940a398f9cd23p-1, 0x1.180996c77c8cap-1, 0x1.f6c118574c83ep-3,
    -0x1.523eb8420f5f5p-4, -0x1.9b560b9f596eap-2, -0x1.5ac4a670a1cffp-1, -0x1.c24a622e3e9f9p-1,
    -0x1.f90459484f2b2p-1, 0x1.0000000000000p+0, 0x1.ed037ea3d2dbbp-1, 0x1.b57675cf309eep-1,
    0x1.5d779b07cfef7p-1, 0x1.d71b4a0c5a6c8p-2, 0x1.a0ad8bd1e2882p-3, -0x1.17855b599f3b9p-4,
    -0x1.56eaae597c776p-2, -0x1.2742a4a775cfbp-1, -0x1.8d2a07c16d46fp-1, -0x1.d59cb83ef99bcp-1,
    -0x1.fb3b3035aa6cdp-1, 0x1.0000000000000p+0, 0x1.f4079c06c0992p-1, 0x1.d0adb9b447ccfp-1,
    0x1.979982a38e65ap-1, 0x1.4b76371208a62p-1, 0x1.dfa67657e7608p-2, 0x1.11f2f2e2f1e3bp-2,
    0x1.bb81853a18977p-5, -0x1.4b545c0234a71p-3, -0x1.7b057f20bf2e4p-2, -0x1.1f53e93956dbfp-1,
    -0x1.73b5ae5db4e10p-1, -0x1.b6b5fbd9f7255p-1, -0x1.e532cbe45c954p-1, -0x1.fcffa67b61650p-1,
    0x1.0000000000000p+0, 0x1.f584f2ce43b84p-1, 0x1.d681a366a00fap-1, 0x1.a43b1b1379affp-1,
    0x1.60c045a2e9729p-1, 0x1.0ed45eea3b09fp-1, 0x1.63a3fcfaca412p-2, 0x1.361fc440b478fp-3,
    -0x1.9eeb01776b57dp-5, -0x1.00ab0eb2d7d94p-2, -0x1.c2f6af3928a8ep-2, -0x1.3965f49174d13p-1,
    -0x1.847bf1d5146ccp-1, -0x1.bfaa5c136b224p-1, -0x1.e884f0cc22cccp-1, -0x1.fd5f830f860f9p-1,
    0x1.0000000000000p+0, 0x1.8836fa2cf5039p-1, 0x1.63a1a7e0b738ap-3, -0x1.0000000000000p-1,
    -0x1.e11f642522d1cp-1,
};
static __constant__ double kTrigSin[89] = {
    0x0.0p+0, 0x1.bb67ae8584caap-1, 0x0.0p+0, 0x1.e6f0e134454ffp-1,
    0x1.2cf2304755a5ep-1, 0x0.0p+0, 0x1.904c37505de4bp-1, 0x1.f329c0558e969p-1,
    0x1.bc4c04d71abc1p-2, 0x0.0p+0, 0x1.14cedf8bb580bp-1, 0x1.d1bb48eee2c13p-1,
    0x1.fac9e043842efp-1, 0x1.82f19bb3a28a1p-1, 0x1.207e7fd768dbfp-2, 0x0.0p+0,
    0x1.dbe064267c47cp-2, 0x1.a55e242a4c3d2p-1, 0x1.fc44566966769p-1, 0x1.deba72ef20147p-1,
    0x1.5384d024c2f84p-1, 0x1.ea1e54bc48dbfp-3, 0x0.0p+0, 0x1.71e955d8e7cdcp-2,
    0x1.58eea2a9d6da3p-1, 0x1.ca52d7c9e640bp-1, 0x1.fdd0deb564b22p-1, 0x1.ec746923c349fp-1,
    0x1.9895b6c9a05f6p-1, 0x1.0d8884363dd80p-1, 0x1.7851aacd6c6b4p-3, 0x0.0p+0,
    0x1.4c7e04850cfaap-2, 0x1.3a7a16b394423p-1, 0x1.aca115aae3de4p-1, 0x1.f0553b4de2e18p-1,
    0x1.fe40529a542aap-1, 0x1.d4e03dd110b08p-1, 0x1.78b0cdee73e0fp-1, 0x1.e75ec0ded7beep-2,
    0x1.5116f7f2d58c5p-3, 0x0.0p+0, 0x1.14459ad2be466p-2, 0x1.0a06e851db7cap-1,
    0x1.763021aaa15dap-1, 0x1.c698e42f47b09p-1, 0x1.f54a827142577p-1, 0x1.fece70dfd3efbp-1,
    0x1.e270060999288p-1, 0x1.a249e0b897ca9p-1, 0x1.431df5838f7efp-1, 0x1.97f6748e524b2p-2,
    0x1.16de8a4564f0ap-3, 0x0.0p+0, 0x1.b8426c12812bcp-3, 0x1.adf7689c97b70p-2,
    0x1.35d9650d47852p-1, 0x1.863a1ada0cfa6p-1, 0x1.c45bb0d10918cp-1, 0x1.ed566cb3dcba1p-1,
    0x1.ff3fc588e859dp-1, 0x1.f941537248537p-1, 0x1.dba2d62cb789fp-1, 0x1.a7c6da34af89fp-1,
    0x1.601a24ba81342p-1, 0x1.07f6acd7cdce2p-1, 0x1.46f6faf5fcb72p-2, 0x1.badb02034d9ffp-4,
    0x0.0p+0, 0x1.9c4266041ca8fp-3, 0x1.93d20572ca90bp-2, 0x1.247d447a27216p-1,
    0x1.73180a4b0d300p-1, 0x1.b2818007c19dfp-1, 0x1.e0210c26a6e6fp-1, 0x1.fa18852c3e08ap-1,
    0x1.ff57c5208ccf9p-1, 0x1.efa7cddb128fap-1, 0x1.cbad095f50378p-1, 0x1.94e08eb13c451p-1,
    0x1.4d80b1ad9ccf6p-1, 0x1.f0f2ff6705becp-2, 0x1.328c3f1b322cbp-2, 0x1.9e62aca53c49fp-4,
    0x0.0p+0, 0x1.491b7523c161dp-1, 0x1.f838b8c811c17p-1, 0x1.bb67ae8584caap-1,
    0x1.5e3a8748a0bf5p-2,
};

}  // namespace so3g
