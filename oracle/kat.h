/*
 * kat.h -- TEST INFRASTRUCTURE ONLY: the known-answer-test interface shared
 * by the three implementations of the reference's unit-level functions:
 *   ref_kat     (oracle/_ref/libref_kat.so: the reference's own headers,
 *                compiled unmodified by oracle/Makefile `ref`),
 *   oracle_kat  (the oracle, oracle/restir_oracle.cpp),
 *   crisb_selftest_kat (the CUDA product's device functions, run on the GPU).
 * One call evaluates function `fn` on n packed input records and writes n
 * packed output records; records are arrays of 32-bit words (64-bit values
 * as two words, low word first).  Layouts, per record:
 */
#ifndef CRISB_KAT_H
#define CRISB_KAT_H

/* SampleTEA64(v0, v1), random.h:24-38.  in: v0, v1.  out: u64 */
#define KAT_TEA64 1
/* PCG32(initstate, initseq), random.h:47-60.  in: u64 initstate, u64 initseq.
 * out: u64 state, u64 inc */
#define KAT_PCG_SEED 2
/* draws from PCG32 {state, inc}: a = NextUint32(), then NextFloat(), then
 * NextUint64(), random.h:62-84.  in: u64 state, u64 inc.
 * out: a, float bits, u64 draw, u64 state after */
#define KAT_PCG_DRAWS 3
/* GetLuminance, luminance.h:6-9.  in: 3 floats.  out: float */
#define KAT_LUMINANCE 4
/* ComputeCanonicalPairwiseMISWeight, path_gen.h:15-31.  in: basis-at-basis
 * rgb, basis-at-neighbour rgb, jacobian, pairwiseK, canonicalM, neighborM
 * (10 floats).  out: float */
#define KAT_MIS_CANON 5
/* ComputeNeighborPairwiseMISWeight, path_gen.h:33-48.  in: neighbour-at-basis
 * rgb, neighbour-at-neighbour rgb, jacobian, pairwiseK, canonicalM, neighborM.
 * out: float */
#define KAT_MIS_NEIGH 6
/* SelectSpatialNeighbor, path_gen.h:50-57, window radius 10
 * (WINDOW_RADIUS, path_gen.h:12).  in: px, py, u64 state, u64 inc.
 * out: nx, ny, u64 state after */
#define KAT_SELECT_NEIGHBOR 7
/* CalcReconnectionJacobian, path_gen.h:59-72.  in: oldXi, newXi, targetPos,
 * targetNormal (12 floats).  out: float */
#define KAT_JACOBIAN 8
/* Reservoir::Update x KAT_RES_STEPS, then FinalizeGRIS, Reservoir.h:28-50.
 * in: u64 state, u64 inc, wSum0, confidence0, f0 rgb (the initial sample),
 * then per step w, inputConfidence, f rgb.
 * out: per step accepted (0/1), wSum, confidence; then the index of the final
 * sample (KAT_RES_STEPS = the initial one), wSum after FinalizeGRIS, u64 state */
#define KAT_RESERVOIR 9
#define KAT_RES_STEPS 8
/* D_GGX, V_SmithJointGGX (brdf.cu:99-112), FresnelSchlick(vec3 F0, VdotH)
 * (brdf.cu:34-37).  in: NdotH, NdotL, NdotV, roughness, VdotH, F0 rgb.
 * out: D, V, F rgb */
#define KAT_GGX 10
/* SpawnCameraRay, Camera.h:14-22.  in: pos, U, V, W (12 floats), viewport x,
 * y.  out: dir (3 floats) */
#define KAT_CAMERA_RAY 11

#define KAT_NUM_FN 11

/* words per input / output record of each function (index = fn) */
#define KAT_IN_WORDS {0, 2, 4, 4, 3, 10, 10, 6, 12, 4 + 2 + 3 + 5 * KAT_RES_STEPS, 8, 14}
#define KAT_OUT_WORDS {0, 2, 4, 6, 1, 1, 1, 4, 1, 3 * KAT_RES_STEPS + 4, 5, 3}

#endif
