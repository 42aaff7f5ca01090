/*
 * clast_oracle.h -- C API of the CPU oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * The oracle is a scalar C++ restatement of the CLAST reference's
 * seed-and-extend path (masayano/CLAST).  Only the test suite, the smoke
 * check and bench.py's CPU-baseline leg may load it, and only as the checker
 * or as the timed CPU baseline -- never as part of the product path.
 *
 * Parity of this restatement is pinned against the reference itself, built
 * for the host CPU by oracle/build_ref.py (see tests/test_oracle_pin.py).
 */
#ifndef CLAST_ORACLE_H_
#define CLAST_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_params {
  int32_t lmer;        /* -lMer   */
  int32_t stride;      /* -stride */
  int32_t cut_repeat;  /* -repeat (-1 = unlimited) */
  int32_t width;       /* -width  */
  int32_t gap;         /* -gap    */
  int32_t local;       /* -local  (0 = global) */
  double cutoff;       /* -cutOff (-1 = none)  */
  double total_db;     /* totalDatabaseSize (CHostSetting.cu:46-58) */
  double K;            /* 0.71 */
  double lambda;       /* 1.37 */
} oracle_params;

/* Structure-of-arrays hit list, allocated by the oracle. */
typedef struct oracle_hits {
  int64_t n;
  int32_t* t_id;
  int32_t* t_idx;
  int32_t* q_id;
  int32_t* q_idx;
  int32_t* t_len;
  int32_t* q_len;
  int32_t* match;
  int32_t* score;
  double* evalue;
} oracle_hits;

/* Stages returned by oracle_window_search. */
enum {
  ORACLE_STAGE_RAW_SEEDS = 1,      /* createRawSeedList output            */
  ORACLE_STAGE_FILTERED_SEEDS = 2, /* after deleteDuplicateSeeds          */
  ORACLE_STAGE_ALIGNED = 3,        /* after alignment + E-value, pre-filter (reference hit order) */
  ORACLE_STAGE_FINAL = 4           /* CDeviceHitList result (A13)         */
};

/* One (target window, query window) pair, the reference's in-process seam
 * CDeviceHashTable + CDeviceSeqList_query + CDeviceHitList
 * (CHostSchedular.cu:141,169,187).  Base arrays include the (l-1)-base joint
 * after every sequence; gateways are window-relative sequence starts; ids of
 * the first sequence are t_begin / q_begin (q_begin even: '+' strands are
 * even ids, '-' strands odd).  Returns 0 or a negative error code. */
int oracle_window_search(const oracle_params* p,
                         const char* t_bases, int64_t t_nbases, const int32_t* t_gateway,
                         const int32_t* t_lengths, int32_t t_nseqs, int32_t t_begin,
                         const char* q_bases, int64_t q_nbases, const int32_t* q_gateway,
                         const int32_t* q_lengths, int32_t q_nseqs, int32_t q_begin,
                         int32_t stage, oracle_hits* out);

void oracle_hits_free(oracle_hits* h);

/* Whole command line, like the reference's `clast` binary (main.cu:16-112):
 * reads FASTA, appends the 10-column TSV to -o.  threads <= 0: OpenMP default.
 * Returns 0 on success, a negative code on a usage or input error (message in
 * oracle_last_error()). */
int oracle_main(int argc, const char** argv, int threads);

const char* oracle_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
