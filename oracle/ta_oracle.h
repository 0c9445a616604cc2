/* Test infrastructure only (the checker, never the product): a CPU restatement
 * in FP64 of the reference's batched indicator path. Each family follows either
 * the vendored TA-Lib 0.8.3 C that the reference pins as its oracle
 * (src/compat/talib08_formulas.inc), or, for families the vendored set lacks,
 * the reference's own kernels/states; the citation sits beside each function in
 * ta_oracle.c. Rows are series-major float32 matrices; outputs are float64 with
 * NaN warm-up (candles: int32 with 0 warm-up).
 *
 * Parity pinning: SMA EMA WMA RSI MACD ATR TRANGE BBANDS STOCH STDDEV VAR
 * LINEARREG DEMA TEMA T3 are pinned against the vendored TA-Lib compiled from the
 * reference tree (oracle/_ref); OBV AD ADOSC MFI NATR and the candle patterns are
 * pinned against the reference's StreamStates.h / CandleUtils.h compiled on the
 * host. RMA is pinned against the vendored TA_RMA (the reference's device path
 * runs that same function) and, bit for bit, against the reference's TA-Lib
 * 0.8.3 fixture tests/fixtures/talib08_typed.json (RMA(close, 14)). IBS and
 * MARKETFI and QSTICK are pinned against the vendored TA_IBS / TA_MARKETFI /
 * TA_QSTICK. ROC ROCP ROCR ROCR100 MOM MEDPRICE TYPPRICE
 * AVGPRICE WCLPRICE MIDPRICE MIDPOINT restate the reference's float kernels
 * (src/indicators/ROC*.cu, Momentum.cu, MedPrice.cu, TypPrice.cu, AvgPrice.cu,
 * WclPrice.cu, MIDPRICE.cu, MIDPOINT.cu) operation for operation. ROC ROCP
 * MEDPRICE TYPPRICE MIDPRICE are pinned against the vendored TA-Lib functions
 * of the same names within the float tolerance; ROCR ROCR100 MOM AVGPRICE
 * WCLPRICE MIDPOINT are not in the vendored set and are pinned by known
 * answers only, as are the NaN-strict rolling statistics (ClubPack.cu). ADX DX CCI WILLR CORREL SUM MIN MAX have no CPU code in
 * the reference: they are pinned by known-answer tests only ("parity partially
 * unpinned").
 */
#ifndef TA_ORACLE_H
#define TA_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum OracleFamily {
  ORC_SMA = 0, ORC_EMA, ORC_WMA, ORC_RSI, ORC_MACD, ORC_ATR, ORC_NATR, ORC_TRANGE,
  ORC_ADX, ORC_DX, ORC_BBANDS, ORC_STOCH, ORC_CCI, ORC_OBV, ORC_AD, ORC_ADOSC,
  ORC_MFI, ORC_WILLR, ORC_SUM, ORC_MIN, ORC_MAX, ORC_STDDEV, ORC_VAR, ORC_LINEARREG,
  ORC_CORREL, ORC_DEMA, ORC_TEMA, ORC_T3, ORC_ROC, ORC_RMA, ORC_MEDPRICE,
  ORC_TYPPRICE, ORC_MIDPRICE, ORC_ROCP, ORC_ROCR, ORC_ROCR100, ORC_MOM,
  ORC_AVGPRICE, ORC_WCLPRICE, ORC_MIDPOINT, ORC_RMEAN, ORC_RMAX, ORC_RMIN,
  ORC_RSTD, ORC_IBS, ORC_MARKETFI, ORC_QSTICK, ORC_AROON, ORC_AROONOSC, ORC_FAMILY_COUNT
};

/* ins: the family's input planes (see oracle/oracle.py INPUTS); outs: its output
 * planes. Row s of every plane starts at s*T. iparams/fparams: periods and real
 * parameters in the family's order. threads<=0 means all cores. Returns 0 or -1
 * for an unknown family / invalid parameter. */
int orc_batch(int family, const float* const* ins, int S, int T,
              const int* iparams, const double* fparams,
              double* const* outs, int threads);

/* Ragged variant: row s spans [offsets[s], offsets[s+1]) of every plane. */
int orc_batch_ragged(int family, const float* const* ins, int S,
                     const long long* offsets, const int* iparams,
                     const double* fparams, double* const* outs, int threads);

/* Candles: the 63 reference families (order of the ct_cdl_*_batch_d
 * declarations); out is int32, 0 in warm-up. */
int orc_cdl_count(void);
int orc_cdl_lookback(int pattern);
int orc_cdl(int pattern, const float* o, const float* h, const float* l,
            const float* c, int S, int T, int* out, int threads);
int orc_cdl_ragged(int pattern, const float* o, const float* h, const float* l,
                   const float* c, int S, const long long* offsets, int* out,
                   int threads);

#ifdef __cplusplus
}
#endif
#endif
