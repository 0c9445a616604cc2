/* tacuda-b200: B200-native (sm_100a) implementation of TACUDA's batched
 * indicator path behind its C ABI.
 *
 * Every declaration below except the ct_b200_* block keeps the name, argument
 * list, argument meaning and status codes of the reference's include/tacuda.h
 * (TACUDA 0.9.3) or include/tacuda_device.h; the comment beside each gives the
 * reference line it replaces. Matrices are series-major (numSeries rows of
 * seriesLen float32, row i contiguous) in device memory owned by the caller.
 * stream == 0 is the legacy default stream: the call is ordered after prior
 * work on it and returns when the batch is done. A non-null stream only
 * enqueues work (no host synchronisation) and, apart from the first call on a
 * device, allocates nothing, so it can be captured in a CUDA graph.
 * maxConcurrency is accepted for compatibility and ignored: every batch call
 * is one kernel launch.
 *
 * The ct_b200_* block is append-only new surface (multi-indicator fused
 * launches, ragged rows through a plan, int32 candles, per-series alpha with
 * its adjoint); the reference has no counterpart for it.
 */
#ifndef TACUDA_B200_H
#define TACUDA_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#if defined(_WIN32)
#define CTAPI_EXPORT __declspec(dllexport)
#else
#define CTAPI_EXPORT __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* include/tacuda.h:32-40 */
typedef enum ctStatus {
  CT_STATUS_SUCCESS = 0,
  CT_STATUS_ALLOC_FAILED = 1,
  CT_STATUS_COPY_FAILED = 2,
  CT_STATUS_KERNEL_FAILED = 3,
  CT_STATUS_INVALID_ARGUMENT = 4,
  CT_STATUS_DEVICE_ERROR = 5,
  CT_STATUS_UNSUPPORTED = 6,
} ctStatus_t;

CTAPI_EXPORT const char* ct_status_string(ctStatus_t status); /* tacuda.h:45 */
CTAPI_EXPORT const char* ct_get_last_error(void);             /* tacuda.h:54 */
CTAPI_EXPORT const char* ct_version(void);                    /* tacuda.h:70 */

/* ---- device batch API (include/tacuda.h:893-2950) ---- */

CTAPI_EXPORT ctStatus_t ct_sma_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:904 */
CTAPI_EXPORT ctStatus_t ct_ema_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:909 */
CTAPI_EXPORT ctStatus_t ct_wma_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:958 */
CTAPI_EXPORT ctStatus_t ct_rsi_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:914 */
CTAPI_EXPORT ctStatus_t ct_atr_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int period, float initial, int maxConcurrency, cudaStream_t stream); /* tacuda.h:919 */
CTAPI_EXPORT ctStatus_t ct_macd_batch_d(const float *d_inputs, float *d_macds, float *d_signals, float *d_hists, int seriesLen, int numSeries, int fastPeriod, int slowPeriod, int signalPeriod, int maType, int maxConcurrency, cudaStream_t stream); /* tacuda.h:926 */
CTAPI_EXPORT ctStatus_t ct_bbands_batch_d(const float *d_inputs, float *d_uppers, float *d_middles, float *d_lowers, int seriesLen, int numSeries, int period, float upperMul, float lowerMul, int maxConcurrency, cudaStream_t stream); /* tacuda.h:933 */
CTAPI_EXPORT ctStatus_t ct_stochastic_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_ks, float *d_ds, int seriesLen, int numSeries, int kPeriod, int dPeriod, int maxConcurrency, cudaStream_t stream); /* tacuda.h:940 */
CTAPI_EXPORT ctStatus_t ct_dema_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:967 */
CTAPI_EXPORT ctStatus_t ct_tema_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:977 */
CTAPI_EXPORT ctStatus_t ct_t3_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, float vFactor, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1169 */
CTAPI_EXPORT ctStatus_t ct_stddev_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1055 */
CTAPI_EXPORT ctStatus_t ct_var_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1065 */
CTAPI_EXPORT ctStatus_t ct_sum_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1074 */
CTAPI_EXPORT ctStatus_t ct_max_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1083 */
CTAPI_EXPORT ctStatus_t ct_min_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1092 */
CTAPI_EXPORT ctStatus_t ct_linearreg_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1101 */
CTAPI_EXPORT ctStatus_t ct_natr_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1180 */
CTAPI_EXPORT ctStatus_t ct_adx_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1194 */
CTAPI_EXPORT ctStatus_t ct_dx_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1221 */
CTAPI_EXPORT ctStatus_t ct_willr_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1262 */
CTAPI_EXPORT ctStatus_t ct_cci_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1276 */
CTAPI_EXPORT ctStatus_t ct_trange_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1288 */
CTAPI_EXPORT ctStatus_t ct_obv_batch_d(const float *d_closes, const float *d_volumes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1440 */
CTAPI_EXPORT ctStatus_t ct_mfi_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, const float *d_volumes, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1453 */
CTAPI_EXPORT ctStatus_t ct_ad_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, const float *d_volumes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1468 */
CTAPI_EXPORT ctStatus_t ct_adosc_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, const float *d_volumes, float *d_outputs, int seriesLen, int numSeries, int fastPeriod, int slowPeriod, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1483 */
CTAPI_EXPORT ctStatus_t ct_correl_batch_d(const float *d_xs, const float *d_ys, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1826 */
CTAPI_EXPORT ctStatus_t ct_roc_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1007 */
CTAPI_EXPORT ctStatus_t ct_rma_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:4110 */
CTAPI_EXPORT ctStatus_t ct_typprice_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1300 */
CTAPI_EXPORT ctStatus_t ct_medprice_batch_d(const float *d_highs, const float *d_lows, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1339 */
CTAPI_EXPORT ctStatus_t ct_midprice_batch_d(const float *d_highs, const float *d_lows, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1727 */
CTAPI_EXPORT ctStatus_t ct_aroon_batch_d(const float *d_highs, const float *d_lows, float *d_aroon_downs, float *d_aroon_ups, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1363 */
CTAPI_EXPORT ctStatus_t ct_aroonosc_batch_d(const float *d_highs, const float *d_lows, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1350 */
CTAPI_EXPORT ctStatus_t ct_rocp_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1016 */
CTAPI_EXPORT ctStatus_t ct_rocr_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1026 */
CTAPI_EXPORT ctStatus_t ct_rocr100_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1036 */
CTAPI_EXPORT ctStatus_t ct_momentum_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:997 */
CTAPI_EXPORT ctStatus_t ct_midpoint_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1516 */
CTAPI_EXPORT ctStatus_t ct_wclprice_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1312 */
CTAPI_EXPORT ctStatus_t ct_change_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1506 */
CTAPI_EXPORT ctStatus_t ct_rolling_mean_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:3157 */
CTAPI_EXPORT ctStatus_t ct_rolling_max_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:3171 */
CTAPI_EXPORT ctStatus_t ct_rolling_min_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:3185 */
CTAPI_EXPORT ctStatus_t ct_rolling_std_batch_d(const float *d_inputs, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:3199 */
CTAPI_EXPORT ctStatus_t ct_ibs_batch_d(const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:3742 */
CTAPI_EXPORT ctStatus_t ct_marketfi_batch_d(const float *d_highs, const float *d_lows, const float *d_volumes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:3932 */
CTAPI_EXPORT ctStatus_t ct_qstick_batch_d(const float *d_opens, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:4096 */
CTAPI_EXPORT ctStatus_t ct_avgprice_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1428 */

/* candlestick patterns: float signal (+-100/+-80/+-200), warm-up 0 */
CTAPI_EXPORT ctStatus_t ct_cdl_doji_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1877 */
CTAPI_EXPORT ctStatus_t ct_cdl_hammer_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1891 */
CTAPI_EXPORT ctStatus_t ct_cdl_inverted_hammer_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1908 */
CTAPI_EXPORT ctStatus_t ct_cdl_bullish_engulfing_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1926 */
CTAPI_EXPORT ctStatus_t ct_cdl_bearish_engulfing_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1944 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_white_soldiers_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1962 */
CTAPI_EXPORT ctStatus_t ct_cdl_abandoned_baby_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1980 */
CTAPI_EXPORT ctStatus_t ct_cdl_advance_block_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:1998 */
CTAPI_EXPORT ctStatus_t ct_cdl_belt_hold_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2015 */
CTAPI_EXPORT ctStatus_t ct_cdl_breakaway_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2031 */
CTAPI_EXPORT ctStatus_t ct_cdl_two_crows_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2047 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_black_crows_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2064 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_inside_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2081 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_outside_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2099 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_line_strike_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2117 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_stars_in_south_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2135 */
CTAPI_EXPORT ctStatus_t ct_cdl_closing_marubozu_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2153 */
CTAPI_EXPORT ctStatus_t ct_cdl_conceal_baby_swallow_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2171 */
CTAPI_EXPORT ctStatus_t ct_cdl_counterattack_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2189 */
CTAPI_EXPORT ctStatus_t ct_cdl_dark_cloud_cover_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2207 */
CTAPI_EXPORT ctStatus_t ct_cdl_doji_star_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2224 */
CTAPI_EXPORT ctStatus_t ct_cdl_dragonfly_doji_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2241 */
CTAPI_EXPORT ctStatus_t ct_cdl_engulfing_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2258 */
CTAPI_EXPORT ctStatus_t ct_cdl_evening_doji_star_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2275 */
CTAPI_EXPORT ctStatus_t ct_cdl_evening_star_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2292 */
CTAPI_EXPORT ctStatus_t ct_cdl_gap_side_side_white_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2310 */
CTAPI_EXPORT ctStatus_t ct_cdl_gravestone_doji_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2328 */
CTAPI_EXPORT ctStatus_t ct_cdl_hanging_man_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2345 */
CTAPI_EXPORT ctStatus_t ct_cdl_harami_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2361 */
CTAPI_EXPORT ctStatus_t ct_cdl_harami_cross_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2377 */
CTAPI_EXPORT ctStatus_t ct_cdl_high_wave_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2394 */
CTAPI_EXPORT ctStatus_t ct_cdl_hikkake_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2410 */
CTAPI_EXPORT ctStatus_t ct_cdl_hikkake_mod_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2426 */
CTAPI_EXPORT ctStatus_t ct_cdl_homing_pigeon_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2444 */
CTAPI_EXPORT ctStatus_t ct_cdl_identical_three_crows_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2462 */
CTAPI_EXPORT ctStatus_t ct_cdl_in_neck_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2479 */
CTAPI_EXPORT ctStatus_t ct_cdl_kicking_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2495 */
CTAPI_EXPORT ctStatus_t ct_cdl_kicking_by_length_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2512 */
CTAPI_EXPORT ctStatus_t ct_cdl_ladder_bottom_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2530 */
CTAPI_EXPORT ctStatus_t ct_cdl_long_legged_doji_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2548 */
CTAPI_EXPORT ctStatus_t ct_cdl_long_line_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2565 */
CTAPI_EXPORT ctStatus_t ct_cdl_marubozu_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2581 */
CTAPI_EXPORT ctStatus_t ct_cdl_matching_low_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2597 */
CTAPI_EXPORT ctStatus_t ct_cdl_mat_hold_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2614 */
CTAPI_EXPORT ctStatus_t ct_cdl_morning_doji_star_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2631 */
CTAPI_EXPORT ctStatus_t ct_cdl_morning_star_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2648 */
CTAPI_EXPORT ctStatus_t ct_cdl_on_neck_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2665 */
CTAPI_EXPORT ctStatus_t ct_cdl_piercing_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2681 */
CTAPI_EXPORT ctStatus_t ct_cdl_rickshaw_man_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2697 */
CTAPI_EXPORT ctStatus_t ct_cdl_rise_fall3_methods_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2715 */
CTAPI_EXPORT ctStatus_t ct_cdl_separating_lines_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2733 */
CTAPI_EXPORT ctStatus_t ct_cdl_shooting_star_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2751 */
CTAPI_EXPORT ctStatus_t ct_cdl_short_line_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2768 */
CTAPI_EXPORT ctStatus_t ct_cdl_spinning_top_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2784 */
CTAPI_EXPORT ctStatus_t ct_cdl_stalled_pattern_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2802 */
CTAPI_EXPORT ctStatus_t ct_cdl_stick_sandwich_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2820 */
CTAPI_EXPORT ctStatus_t ct_cdl_takuri_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2836 */
CTAPI_EXPORT ctStatus_t ct_cdl_tasuki_gap_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2852 */
CTAPI_EXPORT ctStatus_t ct_cdl_thrusting_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2868 */
CTAPI_EXPORT ctStatus_t ct_cdl_tristar_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2884 */
CTAPI_EXPORT ctStatus_t ct_cdl_unique_3_river_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2901 */
CTAPI_EXPORT ctStatus_t ct_cdl_upside_gap_2_crows_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2919 */
CTAPI_EXPORT ctStatus_t ct_cdl_xside_gap_3_methods_batch_d(const float *d_opens, const float *d_highs, const float *d_lows, const float *d_closes, float *d_outputs, int seriesLen, int numSeries, int maxConcurrency, cudaStream_t stream); /* tacuda.h:2937 */

/* ---- single-series device API (include/tacuda_device.h:130-540) ---- */
CTAPI_EXPORT ctStatus_t ct_sma_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:130 */
CTAPI_EXPORT ctStatus_t ct_ema_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:136 */
CTAPI_EXPORT ctStatus_t ct_wma_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:142 */
CTAPI_EXPORT ctStatus_t ct_dema_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:145 */
CTAPI_EXPORT ctStatus_t ct_tema_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:148 */
CTAPI_EXPORT ctStatus_t ct_t3_d(const float* d_input, float* d_output, int size, int period, float vFactor, cudaStream_t stream); /* tacuda_device.h:158 */
CTAPI_EXPORT ctStatus_t ct_rsi_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:165 */
CTAPI_EXPORT ctStatus_t ct_atr_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, int period, float percentile, cudaStream_t stream); /* tacuda_device.h:193 */
CTAPI_EXPORT ctStatus_t ct_natr_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:203 */
CTAPI_EXPORT ctStatus_t ct_trange_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:207 */
CTAPI_EXPORT ctStatus_t ct_adx_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:215 */
CTAPI_EXPORT ctStatus_t ct_dx_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:223 */
CTAPI_EXPORT ctStatus_t ct_macd_d(const float* d_input, float* d_macd, float* d_signal, float* d_hist, int size, int fastPeriod, int slowPeriod, int signalPeriod, int maType, cudaStream_t stream); /* tacuda_device.h:239 */
CTAPI_EXPORT ctStatus_t ct_stochastic_d(const float* d_high, const float* d_low, const float* d_close, float* d_slowK, float* d_slowD, int size, int kPeriod, int dPeriod, cudaStream_t stream); /* tacuda_device.h:251 */
CTAPI_EXPORT ctStatus_t ct_willr_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:262 */
CTAPI_EXPORT ctStatus_t ct_cci_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:266 */
CTAPI_EXPORT ctStatus_t ct_bbands_d(const float* d_input, float* d_upper, float* d_middle, float* d_lower, int size, int period, float nbDevUp, float nbDevDn, cudaStream_t stream); /* tacuda_device.h:279 */
CTAPI_EXPORT ctStatus_t ct_ad_d(const float* d_high, const float* d_low, const float* d_close, const float* d_volume, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:298 */
CTAPI_EXPORT ctStatus_t ct_adosc_d(const float* d_high, const float* d_low, const float* d_close, const float* d_volume, float* d_output, int size, int fastPeriod, int slowPeriod, cudaStream_t stream); /* tacuda_device.h:302 */
CTAPI_EXPORT ctStatus_t ct_obv_d(const float* d_close, const float* d_volume, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:307 */
CTAPI_EXPORT ctStatus_t ct_mfi_d(const float* d_high, const float* d_low, const float* d_close, const float* d_volume, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:310 */
CTAPI_EXPORT ctStatus_t ct_stddev_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:319 */
CTAPI_EXPORT ctStatus_t ct_var_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:322 */
CTAPI_EXPORT ctStatus_t ct_sum_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:325 */
CTAPI_EXPORT ctStatus_t ct_max_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:328 */
CTAPI_EXPORT ctStatus_t ct_min_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:331 */
CTAPI_EXPORT ctStatus_t ct_linearreg_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:357 */
CTAPI_EXPORT ctStatus_t ct_correl_d(const float* d_x, const float* d_y, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:540 */
CTAPI_EXPORT ctStatus_t ct_roc_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:174 */
CTAPI_EXPORT ctStatus_t ct_medprice_d(const float* d_high, const float* d_low, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:342 */
CTAPI_EXPORT ctStatus_t ct_typprice_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:345 */
CTAPI_EXPORT ctStatus_t ct_midprice_d(const float* d_high, const float* d_low, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:511 */
CTAPI_EXPORT ctStatus_t ct_aroon_d(const float* d_high, const float* d_low, float* d_aroonDown, float* d_aroonUp, int size, int period, cudaStream_t stream); /* tacuda_device.h:376 */
CTAPI_EXPORT ctStatus_t ct_aroonosc_d(const float* d_high, const float* d_low, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:380 */
CTAPI_EXPORT ctStatus_t ct_rma_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:1212 */
CTAPI_EXPORT ctStatus_t ct_rocp_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:177 */
CTAPI_EXPORT ctStatus_t ct_rocr_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:180 */
CTAPI_EXPORT ctStatus_t ct_rocr100_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:183 */
CTAPI_EXPORT ctStatus_t ct_momentum_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:171 */
CTAPI_EXPORT ctStatus_t ct_midpoint_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:447 */
CTAPI_EXPORT ctStatus_t ct_wclprice_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:349 */
CTAPI_EXPORT ctStatus_t ct_change_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:444 */
CTAPI_EXPORT ctStatus_t ct_rolling_mean_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:981 */
CTAPI_EXPORT ctStatus_t ct_rolling_max_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:985 */
CTAPI_EXPORT ctStatus_t ct_rolling_min_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:988 */
CTAPI_EXPORT ctStatus_t ct_rolling_std_d(const float* d_input, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:991 */
CTAPI_EXPORT ctStatus_t ct_ibs_d(const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:1120 */
CTAPI_EXPORT ctStatus_t ct_marketfi_d(const float* d_high, const float* d_low, const float* d_volume, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:1169 */
CTAPI_EXPORT ctStatus_t ct_qstick_d(const float* d_open, const float* d_close, float* d_output, int size, int period, cudaStream_t stream); /* tacuda_device.h:1209 */
CTAPI_EXPORT ctStatus_t ct_avgprice_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:338 */
CTAPI_EXPORT ctStatus_t ct_cdl_doji_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:555 */
CTAPI_EXPORT ctStatus_t ct_cdl_hammer_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:559 */
CTAPI_EXPORT ctStatus_t ct_cdl_inverted_hammer_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:565 */
CTAPI_EXPORT ctStatus_t ct_cdl_bullish_engulfing_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:571 */
CTAPI_EXPORT ctStatus_t ct_cdl_bearish_engulfing_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:577 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_white_soldiers_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:583 */
CTAPI_EXPORT ctStatus_t ct_cdl_abandoned_baby_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:590 */
CTAPI_EXPORT ctStatus_t ct_cdl_advance_block_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:596 */
CTAPI_EXPORT ctStatus_t ct_cdl_belt_hold_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:602 */
CTAPI_EXPORT ctStatus_t ct_cdl_breakaway_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:608 */
CTAPI_EXPORT ctStatus_t ct_cdl_two_crows_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:614 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_black_crows_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:620 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_inside_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:626 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_outside_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:632 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_line_strike_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:638 */
CTAPI_EXPORT ctStatus_t ct_cdl_three_stars_in_south_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:644 */
CTAPI_EXPORT ctStatus_t ct_cdl_closing_marubozu_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:651 */
CTAPI_EXPORT ctStatus_t ct_cdl_conceal_baby_swallow_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:657 */
CTAPI_EXPORT ctStatus_t ct_cdl_counterattack_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:664 */
CTAPI_EXPORT ctStatus_t ct_cdl_dark_cloud_cover_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:670 */
CTAPI_EXPORT ctStatus_t ct_cdl_doji_star_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:676 */
CTAPI_EXPORT ctStatus_t ct_cdl_dragonfly_doji_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:682 */
CTAPI_EXPORT ctStatus_t ct_cdl_engulfing_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:688 */
CTAPI_EXPORT ctStatus_t ct_cdl_evening_doji_star_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:694 */
CTAPI_EXPORT ctStatus_t ct_cdl_evening_star_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:700 */
CTAPI_EXPORT ctStatus_t ct_cdl_gap_side_side_white_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:706 */
CTAPI_EXPORT ctStatus_t ct_cdl_gravestone_doji_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:712 */
CTAPI_EXPORT ctStatus_t ct_cdl_hanging_man_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:718 */
CTAPI_EXPORT ctStatus_t ct_cdl_harami_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:724 */
CTAPI_EXPORT ctStatus_t ct_cdl_harami_cross_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:730 */
CTAPI_EXPORT ctStatus_t ct_cdl_high_wave_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:736 */
CTAPI_EXPORT ctStatus_t ct_cdl_hikkake_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:742 */
CTAPI_EXPORT ctStatus_t ct_cdl_hikkake_mod_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:748 */
CTAPI_EXPORT ctStatus_t ct_cdl_homing_pigeon_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:754 */
CTAPI_EXPORT ctStatus_t ct_cdl_identical_three_crows_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:760 */
CTAPI_EXPORT ctStatus_t ct_cdl_in_neck_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:767 */
CTAPI_EXPORT ctStatus_t ct_cdl_kicking_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:773 */
CTAPI_EXPORT ctStatus_t ct_cdl_kicking_by_length_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:779 */
CTAPI_EXPORT ctStatus_t ct_cdl_ladder_bottom_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:785 */
CTAPI_EXPORT ctStatus_t ct_cdl_long_legged_doji_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:791 */
CTAPI_EXPORT ctStatus_t ct_cdl_long_line_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:797 */
CTAPI_EXPORT ctStatus_t ct_cdl_marubozu_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:803 */
CTAPI_EXPORT ctStatus_t ct_cdl_matching_low_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:809 */
CTAPI_EXPORT ctStatus_t ct_cdl_mat_hold_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:815 */
CTAPI_EXPORT ctStatus_t ct_cdl_morning_doji_star_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:821 */
CTAPI_EXPORT ctStatus_t ct_cdl_morning_star_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:827 */
CTAPI_EXPORT ctStatus_t ct_cdl_on_neck_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:833 */
CTAPI_EXPORT ctStatus_t ct_cdl_piercing_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:839 */
CTAPI_EXPORT ctStatus_t ct_cdl_rickshaw_man_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:845 */
CTAPI_EXPORT ctStatus_t ct_cdl_rise_fall3_methods_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:851 */
CTAPI_EXPORT ctStatus_t ct_cdl_separating_lines_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:857 */
CTAPI_EXPORT ctStatus_t ct_cdl_shooting_star_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:863 */
CTAPI_EXPORT ctStatus_t ct_cdl_short_line_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:869 */
CTAPI_EXPORT ctStatus_t ct_cdl_spinning_top_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:875 */
CTAPI_EXPORT ctStatus_t ct_cdl_stalled_pattern_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:881 */
CTAPI_EXPORT ctStatus_t ct_cdl_stick_sandwich_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:887 */
CTAPI_EXPORT ctStatus_t ct_cdl_takuri_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:893 */
CTAPI_EXPORT ctStatus_t ct_cdl_tasuki_gap_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:899 */
CTAPI_EXPORT ctStatus_t ct_cdl_thrusting_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:905 */
CTAPI_EXPORT ctStatus_t ct_cdl_tristar_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:911 */
CTAPI_EXPORT ctStatus_t ct_cdl_unique_3_river_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:917 */
CTAPI_EXPORT ctStatus_t ct_cdl_upside_gap_2_crows_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:923 */
CTAPI_EXPORT ctStatus_t ct_cdl_xside_gap_3_methods_d(const float* d_open, const float* d_high, const float* d_low, const float* d_close, float* d_output, int size, cudaStream_t stream); /* tacuda_device.h:929 */

/* ---- host batch API (include/tacuda.h:848-890): host matrices, staged
 * through device memory on the given stream (stream 0: synchronous) ---- */
CTAPI_EXPORT ctStatus_t ct_sma_batch(const float *host_inputs, float *host_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:848 */
CTAPI_EXPORT ctStatus_t ct_ema_batch(const float *host_inputs, float *host_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:853 */
CTAPI_EXPORT ctStatus_t ct_rsi_batch(const float *host_inputs, float *host_outputs, int seriesLen, int numSeries, int period, int maxConcurrency, cudaStream_t stream); /* tacuda.h:858 */
CTAPI_EXPORT ctStatus_t ct_atr_batch(const float *host_highs, const float *host_lows, const float *host_closes, float *host_outputs, int seriesLen, int numSeries, int period, float initial, int maxConcurrency, cudaStream_t stream); /* tacuda.h:863 */
CTAPI_EXPORT ctStatus_t ct_macd_batch(const float *host_inputs, float *host_macds, float *host_signals, float *host_hists, int seriesLen, int numSeries, int fastPeriod, int slowPeriod, int signalPeriod, int maType, int maxConcurrency, cudaStream_t stream); /* tacuda.h:870 */
CTAPI_EXPORT ctStatus_t ct_bbands_batch(const float *host_inputs, float *host_uppers, float *host_middles, float *host_lowers, int seriesLen, int numSeries, int period, float upperMul, float lowerMul, int maxConcurrency, cudaStream_t stream); /* tacuda.h:877 */
CTAPI_EXPORT ctStatus_t ct_stochastic_batch(const float *host_highs, const float *host_lows, const float *host_closes, float *host_ks, float *host_ds, int seriesLen, int numSeries, int kPeriod, int dPeriod, int maxConcurrency, cudaStream_t stream); /* tacuda.h:885 */

/* ---- batch streams (include/tacuda_stream.h:155-269): one handle advances
 * numSeries series of one indicator by n bars per append; the appends' outputs
 * equal one batch call over the concatenated bars. Host matrices, series-major
 * (series s's n bars at [s*n, s*n+n)). Every append runs on the GPU. ---- */
typedef struct ctStreamBatch ctStreamBatch_t;
typedef enum ctStreamExec {
  CT_STREAM_EXEC_AUTO = 0,
  CT_STREAM_EXEC_CPU = 1,
  CT_STREAM_EXEC_GPU = 2,
} ctStreamExec_t;                                                                       /* tacuda_stream.h:180 */
CTAPI_EXPORT ctStatus_t ct_stream_batch_destroy(ctStreamBatch_t *batch);                 /* tacuda_stream.h:186 */
CTAPI_EXPORT ctStatus_t ct_stream_batch_reset(ctStreamBatch_t *batch);                   /* tacuda_stream.h:187 */
CTAPI_EXPORT ctStatus_t ct_stream_batch_lookback(const ctStreamBatch_t *batch, int *outLookback); /* tacuda_stream.h:188 */
CTAPI_EXPORT ctStatus_t ct_stream_batch_series(const ctStreamBatch_t *batch, int *outSeries);     /* tacuda_stream.h:190 */
CTAPI_EXPORT ctStatus_t ct_stream_batch_outputs(const ctStreamBatch_t *batch, int *outCount);     /* tacuda_stream.h:192 */
CTAPI_EXPORT ctStatus_t ct_stream_batch_bars(const ctStreamBatch_t *batch, long long *outBars);    /* tacuda_stream.h:194 */
/* CT_STREAM_EXEC_CPU returns CT_STATUS_UNSUPPORTED: appends always run on the GPU. */
CTAPI_EXPORT ctStatus_t ct_stream_batch_set_exec(ctStreamBatch_t *batch, ctStreamExec_t exec);    /* tacuda_stream.h:196 */
CTAPI_EXPORT ctStatus_t ct_sma_stream_batch_create(int period, int numSeries, ctStreamBatch_t **outBatch);  /* tacuda_stream.h:199 */
CTAPI_EXPORT ctStatus_t ct_ema_stream_batch_create(int period, int numSeries, ctStreamBatch_t **outBatch);  /* tacuda_stream.h:201 */
CTAPI_EXPORT ctStatus_t ct_wma_stream_batch_create(int period, int numSeries, ctStreamBatch_t **outBatch);  /* tacuda_stream.h:203 */
CTAPI_EXPORT ctStatus_t ct_rsi_stream_batch_create(int period, int numSeries, ctStreamBatch_t **outBatch);  /* tacuda_stream.h:205 */
CTAPI_EXPORT ctStatus_t ct_atr_stream_batch_create(int period, int numSeries, ctStreamBatch_t **outBatch);  /* tacuda_stream.h:207 */
CTAPI_EXPORT ctStatus_t ct_natr_stream_batch_create(int period, int numSeries, ctStreamBatch_t **outBatch); /* tacuda_stream.h:209 */
CTAPI_EXPORT ctStatus_t ct_obv_stream_batch_create(int numSeries, ctStreamBatch_t **outBatch);              /* tacuda_stream.h:211 */
CTAPI_EXPORT ctStatus_t ct_ad_stream_batch_create(int numSeries, ctStreamBatch_t **outBatch);               /* tacuda_stream.h:213 */
CTAPI_EXPORT ctStatus_t ct_macd_stream_batch_create(int fastPeriod, int slowPeriod, int signalPeriod, int numSeries, ctStreamBatch_t **outBatch); /* tacuda_stream.h:215 */
CTAPI_EXPORT ctStatus_t ct_bbands_stream_batch_create(int period, float upperMul, float lowerMul, int numSeries, ctStreamBatch_t **outBatch);    /* tacuda_stream.h:218 */
CTAPI_EXPORT ctStatus_t ct_sma_stream_batch_append(ctStreamBatch_t *batch, const float *closes, int n, float *outs);  /* tacuda_stream.h:222 */
CTAPI_EXPORT ctStatus_t ct_ema_stream_batch_append(ctStreamBatch_t *batch, const float *closes, int n, float *outs);  /* tacuda_stream.h:225 */
CTAPI_EXPORT ctStatus_t ct_wma_stream_batch_append(ctStreamBatch_t *batch, const float *closes, int n, float *outs);  /* tacuda_stream.h:228 */
CTAPI_EXPORT ctStatus_t ct_rsi_stream_batch_append(ctStreamBatch_t *batch, const float *closes, int n, float *outs);  /* tacuda_stream.h:231 */
CTAPI_EXPORT ctStatus_t ct_atr_stream_batch_append(ctStreamBatch_t *batch, const float *highs, const float *lows, const float *closes, int n, float *outs);  /* tacuda_stream.h:234 */
CTAPI_EXPORT ctStatus_t ct_natr_stream_batch_append(ctStreamBatch_t *batch, const float *highs, const float *lows, const float *closes, int n, float *outs); /* tacuda_stream.h:239 */
CTAPI_EXPORT ctStatus_t ct_obv_stream_batch_append(ctStreamBatch_t *batch, const float *closes, const float *volumes, int n, float *outs);                   /* tacuda_stream.h:244 */
CTAPI_EXPORT ctStatus_t ct_ad_stream_batch_append(ctStreamBatch_t *batch, const float *highs, const float *lows, const float *closes, const float *volumes, int n, float *outs); /* tacuda_stream.h:248 */
CTAPI_EXPORT ctStatus_t ct_macd_stream_batch_append(ctStreamBatch_t *batch, const float *closes, int n, float *outMacd, float *outSignal, float *outHist);  /* tacuda_stream.h:254 */
CTAPI_EXPORT ctStatus_t ct_bbands_stream_batch_append(ctStreamBatch_t *batch, const float *closes, int n, float *outUpper, float *outMiddle, float *outLower); /* tacuda_stream.h:259 */

/* ========================================================================
 * ct_b200_*: new surface with no counterpart in the reference.
 * ======================================================================== */

/* Families of a fused job (same arithmetic as the matching ct_*_batch_d). */
typedef enum ctB200Family {
  CT_B200_SMA = 0, CT_B200_EMA, CT_B200_WMA, CT_B200_RSI, CT_B200_MACD, CT_B200_ATR,
  CT_B200_NATR, CT_B200_TRANGE, CT_B200_ADX, CT_B200_DX, CT_B200_BBANDS, CT_B200_STOCH,
  CT_B200_CCI, CT_B200_OBV, CT_B200_AD, CT_B200_ADOSC, CT_B200_MFI, CT_B200_WILLR,
  CT_B200_SUM, CT_B200_MIN, CT_B200_MAX, CT_B200_STDDEV, CT_B200_VAR, CT_B200_LINEARREG,
  CT_B200_CORREL, CT_B200_DEMA, CT_B200_TEMA, CT_B200_T3, CT_B200_CDL,
  CT_B200_ROC, CT_B200_RMA, CT_B200_MEDPRICE, CT_B200_TYPPRICE, CT_B200_MIDPRICE,
  CT_B200_ROCP, CT_B200_ROCR, CT_B200_ROCR100, CT_B200_MOM, CT_B200_AVGPRICE, CT_B200_WCLPRICE,
  CT_B200_MIDPOINT, CT_B200_ROLLING_MEAN, CT_B200_ROLLING_MAX, CT_B200_ROLLING_MIN, CT_B200_ROLLING_STD,
  CT_B200_IBS, CT_B200_MARKETFI, CT_B200_QSTICK, CT_B200_AROON, CT_B200_AROONOSC
} ctB200Family_t;

/* Input planes of a batch. */
typedef enum ctB200Plane {
  CT_B200_OPEN = 0, CT_B200_HIGH, CT_B200_LOW, CT_B200_CLOSE, CT_B200_VOLUME, CT_B200_AUX
} ctB200Plane_t;

/* The batch's input planes (device pointers; unused planes may be NULL).
 * Uniform rows: offsets == NULL, numSeries rows of seriesLen bars. Ragged rows
 * (plans only): row s spans [offsets[s], offsets[s+1]) of every plane. */
typedef struct ctB200Series {
  const float* planes[6];
  const int64_t* offsets;
  int64_t seriesLen;
  int numSeries;
} ctB200Series;

/* One indicator of a fused launch. params/fparams follow the argument order of
 * the family's ct_*_batch_d (e.g. MACD: fast, slow, signal; BBANDS: period and
 * fparams up, down; STOCH: kPeriod, dPeriod; T3: period, fparams vFactor;
 * STDDEV: period, fparams nbDev). inputs[] maps the family's inputs to planes;
 * a negative first entry selects the defaults (close; high, low, close;
 * high, low, close, volume; close, volume for OBV; close, aux for CORREL).
 * outputs[] are float32 matrices laid out like the planes. CDL: cdl_mask bit k
 * selects pattern k (order of the ct_cdl_*_batch_d declarations above), written
 * to outputs[0] + k * cdl_stride elements, as int32 when cdl_int32 != 0. */
typedef struct ctB200Job {
  int family;
  int params[3];
  double fparams[2];
  int inputs[4];
  void* outputs[3];
  uint64_t cdl_mask;
  int64_t cdl_stride;
  int cdl_int32;
  /* Arithmetic of SMA SUM WMA BBANDS STDDEV VAR LINEARREG CORREL EMA:
   * 0 FP64 (default), 1 plain FP32, 2 compensated FP32 (float pairs with
   * two-sum / two-product), 3 FP32 per bar with FP64 carries between lanes and
   * tiles (EMA; the windows carry nothing). Other families accept only 0. All
   * jobs of one launch use the same precision. */
  int precision;
} ctB200Job;

/* Evaluate all jobs over a uniform batch in one kernel launch. */
CTAPI_EXPORT ctStatus_t ct_b200_fused_batch_d(const ctB200Series* series, const ctB200Job* jobs,
                                              int numJobs, cudaStream_t stream);

/* Host-memory variant: planes and outputs are host pointers; the call copies
 * inputs in, launches once and copies outputs back on `stream` (stream 0:
 * returns when done). */
CTAPI_EXPORT ctStatus_t ct_b200_fused_batch(const ctB200Series* hostSeries, const ctB200Job* hostJobs,
                                            int numJobs, cudaStream_t stream);

/* Plans: a reusable schedule for a (possibly ragged) batch and job set. Creating
 * a plan may allocate and copy (series order, tuned launch shape); executing
 * one only launches, so executions can be captured in CUDA graphs. The job
 * families and parameters at execution must match those at creation; output
 * and input pointers may change. hostOffsets: numSeries+1 row starts on the
 * host (NULL for uniform rows of seriesLen). */
typedef struct ctB200Plan ctB200Plan;
CTAPI_EXPORT ctStatus_t ct_b200_plan_create(const ctB200Job* jobs, int numJobs, const int64_t* hostOffsets,
                                            int numSeries, int64_t seriesLen, ctB200Plan** plan);
CTAPI_EXPORT ctStatus_t ct_b200_plan_execute(const ctB200Plan* plan, const ctB200Series* series,
                                             const ctB200Job* jobs, int numJobs, cudaStream_t stream);
CTAPI_EXPORT ctStatus_t ct_b200_plan_destroy(ctB200Plan* plan);
/* Time the candidate launch shapes of a plan on the given data and keep the
 * fastest (also stored in the autotuner cache). Synchronises `stream`. */
CTAPI_EXPORT ctStatus_t ct_b200_plan_autotune(ctB200Plan* plan, const ctB200Series* series,
                                              const ctB200Job* jobs, int numJobs, cudaStream_t stream);
/* Launch shape chosen by a plan: engine (0 warp-scan: a warp per series,
 * 1 row-parallel: a CTA per 32 series, 2 look-back: a warp per tile), bars per
 * lane, warps per block, block cap (0 = as many as fit). Null outputs are
 * skipped. */
CTAPI_EXPORT ctStatus_t ct_b200_plan_describe(const ctB200Plan* plan, int* engine, int* barsPerLane,
                                              int* warpsPerBlock, int* blocks);
/* Candidates the last ct_b200_plan_autotune timed: up to maxOut entries of
 * engine, bars per lane, warps per block and milliseconds per launch (null
 * arrays are skipped). Returns how many it timed (0 before any autotune). */
CTAPI_EXPORT int ct_b200_plan_candidates(const ctB200Plan* plan, int maxOut, int* engine, int* barsPerLane,
                                         int* warpsPerBlock, float* ms);
/* Row-parallel engine layout of a plan: the partitions its job set is split
 * into (one grid row each) and the 32-row groups each CTA runs; 0 = the
 * library's default for the job set. Null outputs are skipped. */
CTAPI_EXPORT ctStatus_t ct_b200_plan_describe_rows(const ctB200Plan* plan, int* parts, int* groups);
/* The same for each candidate of the last autotune, in the order of
 * ct_b200_plan_candidates (0 for candidates of the other engines). */
CTAPI_EXPORT int ct_b200_plan_candidates_rows(const ctB200Plan* plan, int maxOut, int* parts, int* groups);

/* All selected candle patterns of a uniform batch in one pass, int32 signals
 * (pattern k of mask at d_out + k * seriesLen * numSeries). */
CTAPI_EXPORT ctStatus_t ct_b200_cdl_batch_d(const float* d_opens, const float* d_highs, const float* d_lows,
                                            const float* d_closes, int32_t* d_out, int seriesLen, int numSeries,
                                            uint64_t patternMask, cudaStream_t stream);
CTAPI_EXPORT int ct_b200_cdl_count(void);
CTAPI_EXPORT const char* ct_b200_cdl_name(int pattern);
CTAPI_EXPORT int ct_b200_cdl_lookback(int pattern);

/* Allocation-free look-back launch (no counterpart in the reference), for
 * callers that cannot allocate memory on the launch path: services that
 * reserve all device memory up front and forbid later growth, latency-critical
 * loops where an allocation (or the pool's first growth) would stall, and code
 * running while the device is fully committed. The jobs of a uniform batch (no
 * candle jobs) run on the look-back engine with their scratch in a static
 * 8 MiB device array per device (held by every GPU that loads the library
 * until exit) instead of the stream-ordered pool; the call makes no cudaMalloc,
 * cudaMallocHost or cudaFree, and on stream 0 it reads the device's error word
 * into a stack variable. The batch must need at most 8 MiB of scratch: 256 B
 * plus 144 B per (round of a row, recurrence stage); larger batches fail with
 * CT_STATUS_INVALID_ARGUMENT. The first call on a device looks up the array's
 * address and must come before any stream capture. Each call zeroes the
 * scratch on its stream before the launch; calls that overlap in time (other
 * streams or threads) race on the one array and must be serialised. On a user
 * stream a bounded wait that ran out is reported by the next synchronous call
 * or by ct_b200_take_device_error. */
CTAPI_EXPORT ctStatus_t ct_b200_fused_lookback_static_d(const ctB200Series* series, const ctB200Job* jobs,
                                                        int numJobs, cudaStream_t stream);

/* Differentiable EMA / MACD / RSI with a continuous smoothing coefficient per
 * series (no counterpart in the reference). Periods fix each indicator's
 * lookback and seed as in TA-Lib; alpha replaces the recurrence coefficient of
 * the EMA, of MACD's fast line and of RSI's Wilder smoothing (alpha = 2/(p+1),
 * resp. 1/p, gives TA-Lib's values within float tolerance). MACD's slow and
 * signal lines keep TA-Lib's 2/(n+1). Inputs must be finite; alpha in (0, 1).
 * The forward pass writes, per series, the recurrence state entering every
 * 256-bar segment into d_checkpoints (ct_b200_alpha_checkpoint_doubles(T)
 * doubles per series); the backward pass reads them instead of per-bar state.
 * Backward: gradients of L = sum(w_ema*EMA + w_macd*MACD + w_signal*SIGNAL +
 * w_hist*HIST + w_rsi*RSI) over the non-warm-up bars with respect to the
 * closes (d_dclose, numSeries x seriesLen) and alpha (d_dalpha, numSeries).
 * Null weight planes count as zero; null forward outputs are skipped. */
typedef struct ctB200AlphaParams {
  int emaPeriod, fastPeriod, slowPeriod, signalPeriod, rsiPeriod;
} ctB200AlphaParams;
CTAPI_EXPORT long long ct_b200_alpha_checkpoint_doubles(int seriesLen);
CTAPI_EXPORT ctStatus_t ct_b200_alpha_forward_d(const float* d_close, const float* d_alpha, int seriesLen,
                                                int numSeries, const ctB200AlphaParams* params, float* d_ema,
                                                float* d_macd, float* d_signal, float* d_hist, float* d_rsi,
                                                double* d_checkpoints, cudaStream_t stream);
CTAPI_EXPORT ctStatus_t ct_b200_alpha_backward_d(const float* d_close, const float* d_alpha, int seriesLen,
                                                 int numSeries, const ctB200AlphaParams* params,
                                                 const double* d_checkpoints, const float* d_w_ema,
                                                 const float* d_w_macd, const float* d_w_signal,
                                                 const float* d_w_hist, const float* d_w_rsi, float* d_dclose,
                                                 float* d_dalpha, cudaStream_t stream);

/* Number of kernel launches this library issued from the calling process
 * (diagnostics; the batch entry points issue one each). */
CTAPI_EXPORT unsigned long long ct_b200_launch_count(void);

/* Errors of asynchronous calls (no counterpart in the reference, whose
 * asynchronous calls report nothing after their launch). Every wait inside
 * this library's kernels is bounded; one that runs out sets an error word of
 * the current device and the kernel returns with outputs that are not valid.
 * Calls with stream == 0 (and the host-matrix calls) read the word after
 * their synchronisation and fail with CT_STATUS_KERNEL_FAILED. For calls on
 * other streams: synchronise them, then this call stores the word in *flags
 * (0: no wait ran out; bit 0: a wait ran out) and clears it. The word is per
 * device, shared by all threads and streams using it. */
CTAPI_EXPORT ctStatus_t ct_b200_take_device_error(int* flags);

#ifdef __cplusplus
}
#endif
#endif /* TACUDA_B200_H */
