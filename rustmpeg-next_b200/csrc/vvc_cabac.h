// Normative CABAC data of ITU-T H.266 clause 9.3 in this repository's layout:
// the context-model initialisation (initId, log2 window size) of every one of
// the 379 contexts for I slices, the first context of each syntax element's
// set, and the small tables of residual coding. Shared by the host-side
// parser of the library and the oracle; tests/test_tables_golden.py compares
// every entry with the reference's literals (cabac.rs CTX_INIT_I and the ctx
// module, residual.rs, cabac.rs RENORM_LPS).
#pragma once
#include <stdint.h>

namespace vvc_cabac {

constexpr int kNumContexts = 379;

// (initId, log2WindowSize) per context, I slices.
constexpr uint8_t kCtxInitI[kNumContexts][2] = {
    {19, 12}, {28, 13}, {38, 8}, {27, 8}, {29, 13}, {38, 12}, {20, 5}, {30, 9},
    {31, 9}, {27, 0}, {6, 8}, {15, 8}, {25, 12}, {19, 12}, {37, 8}, {43, 9},
    {42, 8}, {29, 9}, {27, 8}, {44, 5}, {36, 12}, {45, 13}, {36, 12}, {45, 13},
    {35, 1}, {35, 0}, {0, 5}, {26, 4}, {28, 8}, {26, 4}, {35, 5}, {35, 5},
    {34, 4}, {35, 4}, {35, 10}, {35, 0}, {35, 5}, {35, 1}, {25, 5}, {60, 8},
    {45, 6}, {13, 1}, {28, 5}, {59, 4}, {27, 9}, {34, 5}, {33, 9}, {49, 10},
    {50, 9}, {25, 6}, {35, 8}, {35, 8}, {35, 0}, {35, 0}, {35, 1}, {35, 4},
    {35, 4}, {35, 0}, {35, 0}, {35, 4}, {35, 4}, {35, 4}, {35, 4}, {35, 4},
    {35, 0}, {35, 0}, {35, 4}, {35, 0}, {35, 1}, {14, 9}, {45, 5}, {19, 1},
    {35, 4}, {1, 1}, {27, 0}, {6, 4}, {52, 1}, {15, 5}, {12, 1}, {5, 8},
    {7, 9}, {12, 5}, {21, 0}, {33, 2}, {28, 1}, {36, 0}, {18, 8}, {31, 5},
    {25, 5}, {15, 8}, {25, 12}, {19, 9}, {28, 9}, {14, 10}, {25, 9}, {20, 9},
    {29, 9}, {30, 10}, {19, 8}, {37, 8}, {30, 8}, {38, 10}, {25, 12}, {27, 12},
    {28, 9}, {37, 13}, {34, 4}, {53, 5}, {53, 8}, {46, 9}, {11, 9}, {38, 13},
    {46, 8}, {54, 8}, {27, 8}, {39, 8}, {39, 8}, {39, 5}, {44, 8}, {39, 0},
    {39, 0}, {39, 0}, {19, 8}, {46, 12}, {38, 12}, {39, 8}, {52, 4}, {39, 0},
    {39, 0}, {39, 0}, {18, 8}, {39, 8}, {39, 8}, {39, 8}, {27, 8}, {39, 0},
    {39, 4}, {39, 4}, {0, 0}, {39, 0}, {39, 0}, {39, 0}, {11, 8}, {39, 8},
    {39, 8}, {39, 8}, {19, 4}, {39, 0}, {39, 0}, {39, 0}, {33, 8}, {25, 9},
    {18, 12}, {26, 13}, {34, 13}, {27, 13}, {25, 10}, {26, 13}, {19, 13}, {42, 13},
    {35, 13}, {33, 13}, {19, 13}, {27, 13}, {35, 13}, {35, 13}, {34, 10}, {42, 13},
    {20, 13}, {43, 13}, {20, 13}, {33, 8}, {25, 12}, {26, 12}, {42, 12}, {19, 13},
    {27, 13}, {26, 13}, {50, 13}, {35, 13}, {20, 13}, {43, 13}, {25, 1}, {1, 5},
    {40, 9}, {25, 9}, {33, 9}, {11, 6}, {17, 5}, {25, 9}, {25, 10}, {18, 10},
    {4, 9}, {17, 9}, {33, 9}, {26, 9}, {19, 9}, {13, 9}, {33, 6}, {19, 8},
    {20, 9}, {28, 9}, {22, 10}, {40, 1}, {9, 5}, {25, 8}, {18, 8}, {26, 9},
    {35, 6}, {25, 6}, {26, 9}, {35, 8}, {28, 8}, {37, 9}, {25, 9}, {25, 5},
    {11, 10}, {27, 13}, {20, 13}, {21, 10}, {33, 9}, {12, 10}, {28, 13}, {21, 13},
    {22, 13}, {34, 9}, {28, 10}, {29, 10}, {29, 10}, {30, 13}, {36, 8}, {29, 9},
    {45, 10}, {30, 10}, {23, 13}, {40, 8}, {33, 8}, {27, 9}, {28, 12}, {21, 12},
    {37, 10}, {36, 5}, {37, 9}, {45, 9}, {38, 9}, {46, 13}, {13, 8}, {5, 5},
    {4, 4}, {21, 5}, {14, 4}, {4, 4}, {6, 5}, {14, 4}, {21, 1}, {11, 0},
    {14, 4}, {7, 1}, {14, 0}, {5, 0}, {11, 0}, {21, 0}, {30, 1}, {22, 0},
    {13, 0}, {42, 0}, {12, 5}, {4, 4}, {3, 4}, {13, 8}, {5, 5}, {4, 8},
    {6, 5}, {13, 5}, {11, 4}, {14, 5}, {6, 5}, {5, 4}, {3, 0}, {14, 5},
    {22, 4}, {6, 1}, {4, 0}, {3, 0}, {6, 1}, {22, 4}, {29, 0}, {20, 0},
    {34, 0}, {12, 6}, {4, 5}, {3, 5}, {42, 12}, {35, 5}, {60, 0}, {13, 4},
    {28, 9}, {52, 9}, {42, 10}, {25, 1}, {42, 5}, {42, 9}, {50, 9}, {37, 6},
    {45, 9}, {30, 10}, {46, 5}, {45, 0}, {38, 9}, {46, 5}, {25, 1}, {9, 1},
    {29, 8}, {0, 0}, {28, 9}, {0, 0}, {33, 9}, {43, 2}, {35, 1}, {35, 5},
    {35, 10}, {35, 8}, {35, 4}, {35, 1}, {35, 13}, {35, 8}, {35, 8}, {35, 0},
    {34, 5}, {35, 0}, {35, 0}, {35, 4}, {62, 0}, {39, 0}, {39, 0}, {54, 4},
    {39, 0}, {39, 0}, {31, 1}, {39, 0}, {39, 0}, {11, 0}, {11, 0}, {46, 0},
    {18, 4}, {30, 1}, {31, 4}, {18, 4}, {30, 1}, {31, 4}, {35, 1}, {17, 1},
    {42, 5}, {36, 8}, {12, 1}, {21, 1}, {35, 0}, {18, 5}, {20, 8}, {38, 8},
    {25, 13}, {28, 13}, {38, 8}, {11, 6}, {35, 8}, {10, 1}, {3, 1}, {3, 1},
    {3, 1}, {11, 4}, {5, 2}, {5, 1}, {14, 6}, {12, 1}, {17, 4}, {46, 4},
    {28, 5}, {25, 8}, {46, 8},
};

// First context of each syntax element's set.
constexpr int kCtxSplitFlag = 0;
constexpr int kCtxSplitQtFlag = 9;
constexpr int kCtxSplitHvFlag = 15;
constexpr int kCtxSplit12Flag = 20;
constexpr int kCtxModeConsFlag = 24;
constexpr int kCtxSkipFlag = 26;
constexpr int kCtxMergeFlag = 29;
constexpr int kCtxRegularMergeFlag = 30;
constexpr int kCtxMergeIdx = 32;
constexpr int kCtxMmvdFlag = 33;
constexpr int kCtxMmvdMergeIdx = 34;
constexpr int kCtxMmvdStepMvpIdx = 35;
constexpr int kCtxPredMode = 36;
constexpr int kCtxMultiRefLineIdx = 38;
constexpr int kCtxIntraLumaMpmFlag = 40;
constexpr int kCtxIntraLumaPlanarFlag = 41;
constexpr int kCtxCclmModeFlag = 43;
constexpr int kCtxCclmModeIdx = 44;
constexpr int kCtxIntraChromaPredMode = 45;
constexpr int kCtxMipFlag = 46;
constexpr int kCtxDeltaQp = 50;
constexpr int kCtxInterDir = 52;
constexpr int kCtxRefPic = 58;
constexpr int kCtxSubblockMergeFlag = 60;
constexpr int kCtxAffineFlag = 63;
constexpr int kCtxAffineType = 66;
constexpr int kCtxAffMergeIdx = 67;
constexpr int kCtxBcwIdx = 68;
constexpr int kCtxMvd = 69;
constexpr int kCtxBdpcmMode = 71;
constexpr int kCtxQtRootCbf = 75;
constexpr int kCtxQtCbfY = 77;
constexpr int kCtxQtCbfCb = 81;
constexpr int kCtxQtCbfCr = 83;
constexpr int kCtxSigCoeffGroupLuma = 86;
constexpr int kCtxSigCoeffGroupChroma = 88;
constexpr int kCtxSigFlagLuma = 90;
constexpr int kCtxSigFlagChroma = 102;
constexpr int kCtxSigFlagLuma1 = 110;
constexpr int kCtxSigFlagChroma1 = 122;
constexpr int kCtxSigFlagLuma2 = 130;
constexpr int kCtxSigFlagChroma2 = 142;
constexpr int kCtxParFlagLuma = 150;
constexpr int kCtxParFlagChroma = 171;
constexpr int kCtxGtx2Luma = 182;
constexpr int kCtxGtx2Chroma = 203;
constexpr int kCtxGtx1Luma = 214;
constexpr int kCtxGtx1Chroma = 235;
constexpr int kCtxLastXLuma = 246;
constexpr int kCtxLastXChroma = 266;
constexpr int kCtxLastYLuma = 269;
constexpr int kCtxLastYChroma = 289;
constexpr int kCtxMvpIdx = 292;
constexpr int kCtxSmvdFlag = 293;
constexpr int kCtxSaoMergeFlag = 294;
constexpr int kCtxSaoTypeIdx = 295;
constexpr int kCtxLfnstIdx = 296;
constexpr int kCtxTransformSkipFlag = 310;
constexpr int kCtxMtsIdx = 312;
constexpr int kCtxIspMode = 316;
constexpr int kCtxSbtFlag = 318;
constexpr int kCtxSbtQuadFlag = 320;
constexpr int kCtxSbtHorFlag = 321;
constexpr int kCtxSbtPosFlag = 324;
constexpr int kCtxChromaQpAdjFlag = 325;
constexpr int kCtxChromaQpAdjIdc = 326;
constexpr int kCtxImvFlag = 327;
constexpr int kCtxAlfCtbFlag = 332;
constexpr int kCtxCtbAlfAlternative = 341;
constexpr int kCtxAlfUseApsFlag = 343;
constexpr int kCtxCcAlfFilterControlFlag = 344;
constexpr int kCtxCiipFlag = 350;
constexpr int kCtxIbcFlag = 351;
constexpr int kCtxJointCbCrFlag = 354;
constexpr int kCtxTsSigCoeffGroup = 357;
constexpr int kCtxTsSigFlag = 360;
constexpr int kCtxTsParFlag = 363;
constexpr int kCtxTsGtxFlag = 364;
constexpr int kCtxTsLrg1Flag = 369;
constexpr int kCtxTsResidualSign = 373;
constexpr int kCtxActFlag = 374;
constexpr int kCtxPltFlag = 375;
constexpr int kCtxPaletteTransposeFlag = 376;

// LPS renormalisation shift by (LPS range >> 3).
constexpr uint8_t kRenormLps[32] = {6, 5, 4, 4, 3, 3, 3, 3, 2, 2, 2, 2, 2, 2, 2, 2,
                                    1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};

// residual_coding: last-position prefix context offsets by log2 size, the
// first position of each last-position group, the group of each position,
// and the Rice parameter by the neighbourhood sum.
constexpr uint8_t kPrefixCtx[8] = {0, 0, 0, 3, 6, 10, 15, 21};
constexpr uint8_t kMinInGroup[14] = {0, 1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96};
constexpr uint8_t kGroupIdx[64] = {0,  1,  2,  3,  4,  4,  5,  5,  6,  6,  6,  6,  7,  7,  7,  7,
                                   8,  8,  8,  8,  8,  8,  8,  8,  9,  9,  9,  9,  9,  9,  9,  9,
                                   10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10,
                                   11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11};
constexpr uint8_t kGoRicePars[32] = {0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 2, 2,
                                     2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 3, 3, 3, 3};

}  // namespace vvc_cabac
