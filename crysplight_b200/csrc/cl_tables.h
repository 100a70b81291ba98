/* Generated by gen_tables.py from exact arithmetic (decimal, 60 digits). */
#pragma once

#define CLM_PIO2_HI 0x1.921fb54442d18p+0  /* 1.5707963267948966 */
#define CLM_PIO2_LO 0x1.1a62633145c07p-54  /* 6.123233995736766e-17 */
#define CLM_2_OVER_PI 0x1.45f306dc9c883p-1  /* 0.6366197723675814 */
#define CLM_LN2 0x1.62e42fefa39efp-1  /* 0.6931471805599453 */

#define CLM_S3 -0x1.5555555555555p-3
#define CLM_S5 0x1.1111111111111p-7
#define CLM_S7 -0x1.a01a01a01a01ap-13
#define CLM_S9 0x1.71de3a556c734p-19
#define CLM_S11 -0x1.ae64567f544e4p-26
#define CLM_S13 0x1.6124613a86d09p-33
#define CLM_S15 -0x1.ae7f3e733b81fp-41
#define CLM_S17 0x1.952c77030ad4ap-49
#define CLM_C2 -0x1.0000000000000p-1
#define CLM_C4 0x1.5555555555555p-5
#define CLM_C6 -0x1.6c16c16c16c17p-10
#define CLM_C8 0x1.a01a01a01a01ap-16
#define CLM_C10 -0x1.27e4fb7789f5cp-22
#define CLM_C12 0x1.1eed8eff8d898p-29
#define CLM_C14 -0x1.93974a8c07c9dp-37
#define CLM_C16 0x1.ae7f3e733b81fp-45

#define CLM_L2 -0x1.0000000000000p-1
#define CLM_L3 0x1.5555555555555p-2
#define CLM_L4 -0x1.0000000000000p-2
#define CLM_L5 0x1.999999999999ap-3
#define CLM_L6 -0x1.5555555555555p-3
#define CLM_L7 0x1.2492492492492p-3
#define CLM_L8 -0x1.0000000000000p-3

#define CLM_LOG_JMIN (-19)
#define CLM_LOG_NTAB 47
/* (1/F_j, ln F_j), F_j = 1 + j/64, j = CLM_LOG_JMIN .. */
#define CLM_LOG_TAB_INIT \
    0x1.6c16c16c16c17p+0, -0x1.68ac83e9c6a14p-2,  /* j = -19 */ \
    0x1.642c8590b2164p+0, -0x1.522ae0738a3d8p-2,  /* j = -18 */ \
    0x1.5c9882b931057p+0, -0x1.3c25277333184p-2,  /* j = -17 */ \
    0x1.5555555555555p+0, -0x1.269621134db92p-2,  /* j = -16 */ \
    0x1.4e5e0a72f0539p+0, -0x1.1178e8227e47cp-2,  /* j = -15 */ \
    0x1.47ae147ae147bp+0, -0x1.f991c6cb3b379p-3,  /* j = -14 */ \
    0x1.4141414141414p+0, -0x1.d1037f2655e7bp-3,  /* j = -13 */ \
    0x1.3b13b13b13b14p+0, -0x1.a93ed3c8ad9e3p-3,  /* j = -12 */ \
    0x1.3521cfb2b78c1p+0, -0x1.823c16551a3c2p-3,  /* j = -11 */ \
    0x1.2f684bda12f68p+0, -0x1.5bf406b543db2p-3,  /* j = -10 */ \
    0x1.29e4129e4129ep+0, -0x1.365fcb0159016p-3,  /* j = -9 */ \
    0x1.2492492492492p+0, -0x1.1178e8227e47cp-3,  /* j = -8 */ \
    0x1.1f7047dc11f70p+0, -0x1.da727638446a2p-4,  /* j = -7 */ \
    0x1.1a7b9611a7b96p+0, -0x1.9335e5d594989p-4,  /* j = -6 */ \
    0x1.15b1e5f75270dp+0, -0x1.4d3115d207eacp-4,  /* j = -5 */ \
    0x1.1111111111111p+0, -0x1.08598b59e3a07p-4,  /* j = -4 */ \
    0x1.0c9714fbcda3bp+0, -0x1.894aa149fb343p-5,  /* j = -3 */ \
    0x1.0842108421084p+0, -0x1.0415d89e74444p-5,  /* j = -2 */ \
    0x1.0410410410410p+0, -0x1.0205658935847p-6,  /* j = -1 */ \
    0x1.0000000000000p+0, 0x0.0p+0,  /* j = 0 */ \
    0x1.f81f81f81f820p-1, 0x1.fc0a8b0fc03e4p-7,  /* j = 1 */ \
    0x1.f07c1f07c1f08p-1, 0x1.f829b0e783300p-6,  /* j = 2 */ \
    0x1.e9131abf0b767p-1, 0x1.77458f632dcfcp-5,  /* j = 3 */ \
    0x1.e1e1e1e1e1e1ep-1, 0x1.f0a30c01162a6p-5,  /* j = 4 */ \
    0x1.dae6076b981dbp-1, 0x1.341d7961bd1d1p-4,  /* j = 5 */ \
    0x1.d41d41d41d41dp-1, 0x1.6f0d28ae56b4cp-4,  /* j = 6 */ \
    0x1.cd85689039b0bp-1, 0x1.a926d3a4ad563p-4,  /* j = 7 */ \
    0x1.c71c71c71c71cp-1, 0x1.e27076e2af2e6p-4,  /* j = 8 */ \
    0x1.c0e070381c0e0p-1, 0x1.0d77e7cd08e59p-3,  /* j = 9 */ \
    0x1.bacf914c1bad0p-1, 0x1.29552f81ff523p-3,  /* j = 10 */ \
    0x1.b4e81b4e81b4fp-1, 0x1.44d2b6ccb7d1ep-3,  /* j = 11 */ \
    0x1.af286bca1af28p-1, 0x1.5ff3070a793d4p-3,  /* j = 12 */ \
    0x1.a98ef606a63bep-1, 0x1.7ab890210d909p-3,  /* j = 13 */ \
    0x1.a41a41a41a41ap-1, 0x1.9525a9cf456b4p-3,  /* j = 14 */ \
    0x1.9ec8e951033d9p-1, 0x1.af3c94e80bff3p-3,  /* j = 15 */ \
    0x1.999999999999ap-1, 0x1.c8ff7c79a9a22p-3,  /* j = 16 */ \
    0x1.948b0fcd6e9e0p-1, 0x1.e27076e2af2e6p-3,  /* j = 17 */ \
    0x1.8f9c18f9c18fap-1, 0x1.fb9186d5e3e2bp-3,  /* j = 18 */ \
    0x1.8acb90f6bf3aap-1, 0x1.0a324e27390e3p-2,  /* j = 19 */ \
    0x1.8618618618618p-1, 0x1.1675cababa60ep-2,  /* j = 20 */ \
    0x1.8181818181818p-1, 0x1.22941fbcf7966p-2,  /* j = 21 */ \
    0x1.7d05f417d05f4p-1, 0x1.2e8e2bae11d31p-2,  /* j = 22 */ \
    0x1.78a4c8178a4c8p-1, 0x1.3a64c556945eap-2,  /* j = 23 */ \
    0x1.745d1745d1746p-1, 0x1.4618bc21c5ec2p-2,  /* j = 24 */ \
    0x1.702e05c0b8170p-1, 0x1.51aad872df82dp-2,  /* j = 25 */ \
    0x1.6c16c16c16c17p-1, 0x1.5d1bdbf5809cap-2,  /* j = 26 */ \
    0x1.6816816816817p-1, 0x1.686c81e9b14afp-2,  /* j = 27 */ \

