/*
 * cother_b200 -- B200-native (sm_100a) search path of COTHER behind a C ABI.
 *
 * One context corresponds to one instance of the reference's per-worker
 * driver class CuBatchProcessing (src/libmycu/cupro/CuBatchProcessing.cuh:47-244):
 * it owns a CUDA stream on one GPU, a GPU-resident database chunk and the
 * working memory of the pipeline
 *
 *   score matrix (profile-profile + SS + DDMS)
 *     -> phase-1 gapped local DP + finalization (pass list)
 *     -> alignment statistics and E-values
 *     -> phase-2 MAP forward/backward/MAP alignment + finalization
 *     -> hit records and alignment strings.
 *
 * Profile data cross the boundary exactly as in the reference: 181 parallel
 * structure-of-arrays field arrays given as begin/end pointer tables
 * (char* pmbeg[181], char* pmend[181]; field order of
 * src/libmycu/cupro/PM2DVectorFields.h:51-87).
 *
 * All functions return 0 on success and a non-zero status otherwise; the
 * message of the last failure on the calling thread is returned by
 * cbp_last_error(). No function terminates the process or traps on the
 * device. A context may be used by one host thread at a time; different
 * contexts are independent (several may share a GPU).
 */
#ifndef COTHER_B200_H
#define COTHER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CBP_NFIELDS 181          /* pmv2DTotFlds */
#define CBP_MAX_DST_VALUES 99    /* MAX_N_IR_DISTANCE_VALUES */
#define CBP_SS_CARD 30           /* cardinality of the SS score table */

/* status codes */
enum {
    CBP_OK = 0,
    CBP_ERR_ARG = 1,       /* invalid argument */
    CBP_ERR_CUDA = 2,      /* CUDA runtime error */
    CBP_ERR_STATE = 3,     /* call out of order (e.g. process before transfer) */
    CBP_ERR_MEMORY = 4,    /* device memory budget exceeded */
    CBP_ERR_LIMIT = 5      /* input beyond a format limit (e.g. length >= 65536) */
};

typedef struct cbp_context cbp_context;

/* Options of the path (src/libpro/srcpro/MOptions.cpp:76-147). */
/* Forms of the profile-profile term (cbp_options.tc_form). */
#define CBP_TC_PLAIN 0    /* FP32 CUDA cores, the reference's operation order */
#define CBP_TC_BF16X3 1   /* tensor cores: BF16 hi/lo split, three products, FP32 accumulate */
#define CBP_TC_TF32X3 2   /* tensor cores: TF32 hi/lo split, three products, FP32 accumulate */

typedef struct cbp_options {
    float ssswgt;     /* SSSWGT: weight of the SS score, [0,1) */
    float cvswgt;     /* CVSWGT: weight of the context-vector term, [0,1); > 0 needs
                       * cbp_set_cvs2s_map and context vectors in the profiles
                       * (the reference's own default is 0.15) */
    float ddmswgt;    /* DDMSWGT: weight of the DDMS score */
    int   dstsegm;    /* DSTSEGM: minimum DDMS segment length */
    int   mapaln;     /* MAPALN: 1 = MAP realignment in phase 2 */
    float minpp;      /* MINPP: minimum posterior probability */
    int   ssemodel;   /* SSEMODEL: statistical significance model (0..2) */
    int   x_uninf;    /* X_UNINF: mask uninformative (X) positions */
    float eval;       /* EVAL: E-value threshold */
    int   nohits;     /* NOHITS */
    int   noalns;     /* NOALNS */
    int   tc_form;    /* CBP_TC_*: how the profile-profile term is computed. The
                       * tensor-core forms recast it, for each database profile,
                       * as the contraction [Lq x 20] x [20 x Ld] of the query's
                       * target frequencies with the profile's frequencies divided
                       * by the mean background (no counterpart in the reference,
                       * which sums the 20 quotients on CUDA cores); results agree
                       * with the plain form within about 1e-6 relative, not bit
                       * for bit. */
    int   autotune;   /* 1: on the first slab of each query-length bin (Lq/64), time
                       * the kernel variants (score-kernel rows per block and
                       * column-ordering window, phase-1 DP warps per block) on a
                       * sample of the slab and keep the fastest (no counterpart in
                       * the reference). Results do not depend on the choice. */
    int   all_codes;  /* 1: the phase-1 DP writes backtrack codes for every database
                       * profile (what cbp_read_btck shows then matches the
                       * reference's matrix everywhere); 0: only for the profiles
                       * whose DP maximum exceeds the score threshold, the only
                       * ones the finalization backtraces -- the others take one
                       * sweep without codes. Results do not depend on it. */
} cbp_options;

/* Fill *opt with the values of the parity configuration:
 * SSSWGT=0.12, CVSWGT=0, DDMSWGT=0.2, DSTSEGM=6, MAPALN=1, MINPP=0.28,
 * SSEMODEL=2, X_UNINF=1, EVAL=10, NOHITS=NOALNS=700; the plain FP32
 * profile-profile form, the kernel tuner on and backtrack codes for the
 * finalization's candidates only. */
void cbp_default_options(cbp_options* opt);

/* Create a context on `device`.
 *   ss_table: the SS score table, CBP_SS_CARD x CBP_SS_CARD floats, full
 *             symmetric (the lower triangle of the reference's env/ssss file);
 *   dev_mem_bytes: device memory the context may use for working buffers
 *             (0 = 70% of the free memory at creation).
 * Replaces CuBatchProcessing::CuBatchProcessing
 * (src/libmycu/cupro/CuBatchProcessing.cuh:50-58; device heap planning of
 * src/libmycu/cupro/CuDeviceMemory.cu:285-588). */
int cbp_create(int device, const cbp_options* opt, const float* ss_table,
               size_t dev_mem_bytes, cbp_context** ctx);

/* Release all resources (CuBatchProcessing::~CuBatchProcessing). */
int cbp_destroy(cbp_context* ctx);

/* Database totals used for E-values: residues and sequences of the WHOLE
 * database, not of the chunk (CuBatchProcessing::SetDbDetails,
 * src/libmycu/cupro/CuBatchProcessing.cuh:73-76). */
int cbp_set_db_details(cbp_context* ctx, uint64_t db_len, size_t n_seqs);

/* Query length used for the length adjustment (SetQueryLen, :78-79). */
int cbp_set_query_len(cbp_context* ctx, size_t query_len);

/* Phase-1 score threshold (SetScoreThreshold, :80-82). */
int cbp_set_score_threshold(cbp_context* ctx, float threshold);

/* log E-value threshold for phase 2 (SetLogEThreshold, :83-85). */
int cbp_set_logE_threshold(cbp_context* ctx, float log_threshold);

/* Upload a database chunk and keep it resident until the next call
 * (CuBatchProcessing::TransferCPMData, :62-71; copy of
 * src/libmycu/cupro/CuDeviceMemory.cu:1095-1139). `pmbeg`/`pmend` are the
 * begin/end pointer tables of the chunk's 181 host field arrays; `szfields`
 * is accepted for interface compatibility and may be NULL. */
int cbp_transfer_chunk(cbp_context* ctx, char* const* pmbeg, char* const* pmend,
                       const size_t* szfields);

/* ------------------------------------------------------------------------
 * Binary profile database files in the reference's format v2.2 (what its
 * db2bin writes: "COTHER profile bin database v2.5"; Db::MakeBin_v2_2,
 * src/libpro/srcpro/Db.cpp:340-385, and BinaryWriteProfile_v2_2,
 * src/libpro/srcpro/PMProfileModel.cpp:1250-1810), replacing the chunk
 * reading of TdDataReader/CuDbReader (src/libmycu/cupro/TdDataReader.cpp:
 * 387-984, CuDbReader.cpp:457-519). The file is mapped, not copied. */
typedef struct cbp_db cbp_db;

/* Open and validate a database file (signature, version, address table,
 * section extents, profile lengths, descriptions). */
int cbp_db_open(const char* path, cbp_db** db);
int cbp_db_close(cbp_db* db);
/* Number of profiles, positions and distance values (the file's header). */
int cbp_db_info(cbp_db* db, uint64_t* nprofiles, uint64_t* npositions, uint64_t* ndistances);
/* The lengths of all profiles (nprofiles ints), for planning chunks. */
int cbp_db_profile_lengths(cbp_db* db, int32_t* lens);
/* Profiles first .. first+count-1 as the 181 begin/end field pointers that
 * cbp_transfer_chunk takes, and their descriptions (descs may be NULL; else
 * count entries). The stored fields point into the mapped file, which is
 * mapped read-only (the pointers are char* only to match cbp_transfer_chunk,
 * which never writes through them); the derived ones (pps2DDist,
 * pmv2DAddrPro, pmv2DAddrCV, pmv2DAddrSS) into buffers of the handle. Valid
 * until the next cbp_db_chunk call or cbp_db_close. */
int cbp_db_chunk(cbp_db* db, uint64_t first, uint64_t count, char** beg, char** end,
                 const char** descs);
/* Write profiles given as a 181-field table (one chunk: all fields of the
 * sizes cbp_transfer_chunk expects) with their descriptions (NULL: empty)
 * to a database file of this format. */
int cbp_db_write(const char* path, char* const* beg, char* const* end, const char* const* descs);

/* Use `owner`'s resident database chunk instead of a copy of one's own (no
 * counterpart in the reference, where each worker transfers its chunk).
 * Several contexts on one device can then search the same resident database
 * at the same time, each on its own stream with its own working memory,
 * which is what a request loop that keeps several queries in flight needs.
 * The chunk lives until its last user transfers another chunk or is
 * destroyed. Both contexts must be on the same device. */
int cbp_share_database(cbp_context* ctx, cbp_context* owner);

/* Free and total device memory of `device` in bytes (cudaMemGetInfo), for
 * callers that divide it between contexts (no counterpart in the
 * reference, whose CuDeviceMemory does the same internally). */
int cbp_device_memory(int device, size_t* free_bytes, size_t* total_bytes);

/* Chunk capacities for a query of `query_len` positions (the read-backs
 * GetCurrentMaxDbPos, GetCurrentMaxNDbPros, GetCurrentMaxDbPosPass2 and
 * GetCurrentMaxNDbProsPass2, src/libmycu/cupro/CuBatchProcessing.cuh:106-111,
 * with which the reference's dispatcher sizes the chunks it reads,
 * src/libmycu/cualn/JobDispatcher.cpp:1054-1067). A chunk fits when its
 * resident copy fits the device memory left beside this context's working
 * budget: with profiles of `expected_profile_length` positions on average
 * (the reference's DEV_EXPCT_DBPROLEN), at most *max_db_pros profiles and
 * *max_db_pos positions. The working memory is planned per slab inside the
 * chunk with every profile allowed to pass phase 1, so the phase-2 limits
 * equal the chunk's. All four are 0 when the budget cannot hold one slab of
 * one such profile for this query. */
int cbp_get_capacities(cbp_context* ctx, size_t query_len, size_t expected_profile_length,
                       size_t* max_db_pos, size_t* max_db_pros, size_t* max_pass2_pos,
                       size_t* max_pass2_pros);

/* The context-vector score map (the reference's CVS2Scores, read from
 * src/env/cvs2s and handed to CuDeviceMemory::CacheCVS2Scores,
 * src/libmycu/cupro/CuDeviceMemory.cu:214-219, 691-740): `card` keys on the
 * grid of halves (keys[i] = (i - s)/2 with s the number of negative keys)
 * and their scores, as the reference's reader leaves them (smoothed). It
 * is required before cbp_process when CVSWGT > 0; the database and query
 * profiles then need their context-vector fields (pmv2DCVentrs,
 * pmv2DCVprior, pmv2DCVnorm2). */
int cbp_set_cvs2s_map(cbp_context* ctx, const float* keys, const float* scores, size_t card);

/* Working device memory that one slab of `positions` database positions
 * takes for a query of `query_len` positions under `opt`: what the slab
 * planner charges against a context's budget (the role of the per-chunk
 * size computation of CuDeviceMemory, src/libmycu/cupro/CuDeviceMemory.cu).
 * Host-only; needs no device. */
int cbp_slab_bytes(const cbp_options* opt, size_t query_len, size_t positions, size_t* bytes);

/* Search one query against the resident chunk
 * (CuBatchProcessing::ProcessScoreMatrix, :87-99). `qpmbeg`/`qpmend` are
 * the pointer tables of the query's field arrays (one profile). The call
 * returns when the results are available through cbp_get_results(). */
int cbp_process(cbp_context* ctx, int query_serial, size_t query_len,
                char* const* qpmbeg, char* const* qpmend);

/* Search several queries against the resident chunk in one pass over its
 * database columns: the queries' rows are stacked into one score matrix per
 * slab (one column-order and one score-kernel launch for all of them), and
 * each query's phase 1 follows in the same CUDA graph; statistics, MAP and
 * the hit order then run per query. Each query's results are what
 * cbp_process would give for it alone (thresholds from EVAL for its own
 * length unless set; cbp_set_query_len applies to single queries only).
 * The result calls (cbp_get_hit_records, cbp_get_alignments,
 * cbp_get_hit_list, cbp_format_hits, cbp_get_search_space) read query 0
 * after the call; cbp_select_query chooses another. The inspection calls
 * (cbp_read_*) see the last query. No counterpart in the reference, which
 * searches one query per ProcessScoreMatrix call
 * (src/libmycu/cualn/DevCommThread.cpp:316-355). */
int cbp_process_batch(cbp_context* ctx, size_t nqueries, const size_t* query_lens,
                      char* const* const* qpmbeg, char* const* const* qpmend);

/* Make query k of the last cbp_process/cbp_process_batch call the one the
 * result calls read; *nqueries (may be NULL) receives the call's number of
 * queries. CBP_ERR_ARG when k is out of range. */
int cbp_select_query(cbp_context* ctx, size_t k, size_t* nqueries);

/* Wait until no work of this context is in flight (WaitForIdleChilds). */
int cbp_wait_idle(cbp_context* ctx);

/* Message of the last failure on the calling thread ("" if none). */
const char* cbp_last_error(void);

/* ------------------------------------------------------------------------
 * Inspection of intermediate results of the last cbp_process() call. They
 * exist for verification and refer to the LAST processed slab of database
 * profiles (see cbp_set_max_slab_positions).
 */

/* Copy the score matrices (query positions x slab positions) to host:
 * scores[r * ld + c] and modscores[r * ld + c] for r < query length and
 * c < *ncols (the number of slab positions, written on return).
 * Either output may be NULL; `first_profile` receives the index of the
 * slab's first profile within the chunk. */
int cbp_read_score_matrix(cbp_context* ctx, float* scores, float* modscores,
                          size_t ld, size_t* ncols, size_t* first_profile);

/* Phase-1 results of the profiles of the last slab (index = profile within
 * the slab): score with correlation bonus, #positive substitution scores,
 * beginning/end coordinates packed (x << 16) | y, and whether the profile
 * passed the score threshold; pass_list receives the slab indices of the
 * passed profiles in ascending order (*npass entries). The records follow
 * FinalizeDPPro (src/libmycu/cudp/CuBatchDP_final.cu:61-292). */
int cbp_read_phase1(cbp_context* ctx, float* score, float* psts, uint32_t* beg,
                    uint32_t* end, int* passed, size_t nmax, size_t* nprof,
                    int* pass_list, size_t* npass);

/* The hit records of the last slab's passed pairs as the statistics stage
 * leaves them (CBP_REC_FLOATS floats each, pass-list order), before the
 * phase-2 finalizer overwrites the positives, coordinates, counts and the
 * per-pair log E-value slot (the reference's dp2alndatbuffers between
 * CalculateAlnStatisticsDevice and the MAP stage,
 * src/libmycu/cupro/CuBatchProcessing.cu:430-480). */
int cbp_read_statistics(cbp_context* ctx, float* recs, size_t nmax, size_t* npass);

/* The precision forms (tc_form != CBP_TC_PLAIN) fit the statistical
 * parameters of each passed pair twice, in FP64 (used for its E-value) and
 * in FP32 (the reference's arithmetic); this returns both for the passed
 * pairs of the last slab, 8 doubles each: lambda, K, H, expected score of
 * the FP64 fit, then the same of the FP32 fit (lambda and the expected score
 * per unscaled score unit). No counterpart in the reference, whose fit is
 * FP32 only (src/libmycu/cuss/CuBatchSS_lambda.cuh:80-330, CuBatchSS_K.cuh,
 * CuBatchSS_entropy.cuh). CBP_ERR_STATE in the plain form. */
int cbp_read_fits(cbp_context* ctx, double* fits, size_t nmax, size_t* npass);

/* Backtrack codes of the last slab's phase-1 DP, btck[r * ld + c]
 * (0 stop, 1 left, 2 up, 3 diagonal; src/libmycu/cudp/CuBatchDP_com.h:101-106). */
int cbp_read_btck(cbp_context* ctx, uint8_t* btck, size_t ld);

/* Columns [first_col, first_col + ncols) of the last slab's matrices, for
 * inspecting a sample of a slab too large to copy whole: scores, modscores
 * (float) and phase-1 backtrack codes (uint8), each [query length][ld] on
 * the host with column 0 = slab column first_col. Any output may be NULL.
 * An inspection call with no counterpart in the reference (its matrices are
 * device-internal); CBP_ERR_ARG when the range leaves the slab. */
int cbp_read_slab_columns(cbp_context* ctx, size_t first_col, size_t ncols, float* scores,
                          float* modscores, uint8_t* btck, size_t ld);

/* The MAP stage's forward + backward log probabilities of the match state
 * (the log of the posterior times Z) of pair `pair` of the last slab's pass
 * list (record order within that slab), fb[r * ld + c] for the query rows r
 * and the profile's columns c; *profile_len (may be NULL) receives the
 * profile's length. Meaningful for the pairs the stage realigned (log
 * E-value at most the threshold; MAPALN=1), of the last query processed.
 * An inspection call with no counterpart in the reference, whose matrix is
 * device-internal (src/libmycu/cumapdp/CuBatchMAPDP_bwd.cu); with fb ==
 * NULL only the length is returned. CBP_ERR_STATE without a realignment. */
int cbp_read_map_fb(cbp_context* ctx, size_t pair, float* fb, size_t ld, size_t* profile_len);

/* Phase-1 score threshold and log E-value threshold from the E-value
 * threshold and the gapped Karlin-Altschul parameters (the [GAPPED_A_1]
 * lambda and K of cother.par); search space = query_len * db_len.
 * Replaces JobDispatcher::CalculateScoreThreshold
 * (src/libmycu/cualn/JobDispatcher.cpp:809-860). */
void cbp_score_threshold(size_t query_len, uint64_t db_len, float evalue,
                         float gapped_lambda, float gapped_k,
                         float* score_threshold, float* log_evalue_threshold);

/* Number of floats of one hit record: the fields of TDP2OutputAlnData
 * (src/libmycu/cuss/CuBatchSS_com.h:45-71) in this order: score,
 * original profile number*, offset in the phase-2 position space*,
 * #positive scores, beginning coords*, end coords*, estimated gapped lambda,
 * estimated gapped K, log E-value, log E-value of the pair, min score, max
 * score, expected score, relative entropy, lambda, K, #identities, #gaps
 * (* = uint32 stored in the float's bits; coordinates packed (x<<16)|y). */
#define CBP_REC_FLOATS 18

/* Hit records of the last cbp_process() call, one per pair that passed
 * phase 1, over all slabs, in database order. With recs == NULL only the
 * count is returned. (The reference hands the same array to its finalizer,
 * src/libmycu/cupro/CuBatchProcessing.cu:599-697.) */
int cbp_get_hit_records(cbp_context* ctx, float* recs, size_t max_records, size_t* nrecords);

/* Alignment strings of the last cbp_process() call: 5 rows (query, middle,
 * target, query SS, target SS) of *length bytes each, copied to
 * rows[r * row_stride]. Hit k (record order) owns bytes
 * [newDst_k + k*Lq, newDst_k + k*Lq + Ld_k + Lq) of every row, with its
 * alignment right-aligned and 0-terminated at the slot's last byte; the
 * alignment length is the int stored in the record's log-E-value-of-pair
 * field after realignment (0 when the pair was not realigned). This is the
 * layout the reference's finalizer reads
 * (src/libmycu/cumapdp/CuBatchMAPDP_map_final.cu:190-330). With rows ==
 * NULL only *length is returned. */
int cbp_get_alignments(cbp_context* ctx, char* rows, size_t row_stride, size_t* length);

/* The hits of the last cbp_process() call that the reference's finalizer
 * reports, in its order: records whose log E-value is at most the log E
 * threshold and that were realigned (alignment length >= 1)
 * (src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp:79-92), sorted by
 * log E-value, smallest first (CuBatchProcessingFinalizer.cpp:283-292; equal
 * values keep database order). The order is computed on the device (a sort
 * of all records' keys at the end of cbp_process). *nhits receives the
 * number of reported hits; order[i] receives the record index of the i-th,
 * for i < min(max_hits, *nhits): the top max_hits hits. With order == NULL
 * only the count is returned. */
int cbp_get_hit_list(cbp_context* ctx, int32_t* order, size_t max_hits, size_t* nhits);

/* Effective search space and length adjustment of the last cbp_process()
 * call (AbstractScoreMatrix::ComputeLengthAdjustment,
 * src/libpro/srcsco/AbstractScoreMatrix.cpp:247-393). */
int cbp_get_search_space(cbp_context* ctx, uint64_t* search_space, size_t* delta_length);

/* ------------------------------------------------------------------------
 * Text output of the results: the finalizer's per-hit text and the writer's
 * per-query report, plain (.out) or JSON (.json), in the reference's layout
 * (CuBatchProcessingFinalizer::CompressResultsPlain/JSON,
 * src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp:35-385 and
 * CuBatchProcessingFinalizerJSON.cpp:35-380; AlnWriter::WriteResultsPlain/
 * JSON, src/libmycu/cualn/AlnWriterPlain.cpp:19-398 and AlnWriterJSON.cpp:
 * 19-429; AlnWriter::MergeResults, src/libmycu/cualn/AlnWriter.cpp:216-256). */
#define CBP_FORMAT_PLAIN 0
#define CBP_FORMAT_JSON  1

typedef struct cbp_format_options {
    int format;     /* CBP_FORMAT_PLAIN or CBP_FORMAT_JSON (the reference's -f) */
    int dsclen;     /* DSCLEN: maximum length of a description (1024) */
    int dscwidth;   /* DSCWIDTH: width at which descriptions wrap (80) */
    int alnwidth;   /* ALNWIDTH: alignment characters per line (60) */
    int show;       /* SHOW: statistics footer of each plain hit record (1) */
} cbp_format_options;

/* The reference's defaults (src/env/options.txt). */
void cbp_default_format_options(cbp_format_options* fo);

/* Per-hit text of the last cbp_process() call, for the hits that
 * cbp_get_hit_list reports and in its order: for each, the annotation line
 * of the summary list, a NUL, the hit record (description, scores,
 * alignment, statistics), a NUL. descs[p] is the description of chunk
 * profile p (NULL: none). With buf == NULL only *used (bytes) and *nhits are
 * set; a buffer smaller than *used gives CBP_ERR_LIMIT. */
int cbp_format_hits(cbp_context* ctx, const cbp_format_options* fo, const char* const* descs,
                    char* buf, size_t cap, size_t* used, size_t* nhits);

/* The same from host data, without a context (the finalizer's inputs). */
typedef struct cbp_hits_input {
    const float* recs;        /* hit records, CBP_REC_FLOATS each (cbp_get_hit_records) */
    size_t nrecs;
    const char* rows;         /* the 5 alignment rows (cbp_get_alignments) */
    size_t row_stride;        /* bytes from one row to the next */
    size_t row_length;        /* bytes of each row */
    const int* prof_len;      /* per chunk profile: length */
    const float* prof_eno;    /* per chunk profile: effective number of observations */
    const uint8_t* prof_ss;   /* per chunk profile: carries SS data (NULL: all do) */
    size_t nprof;
    const char* const* descs; /* per chunk profile: description (NULL: none) */
    int query_len;
    float query_eno;
    int query_ss;             /* the query carries SS data */
    float ssswgt;             /* SSSWGT > 0 shows the SS rows of plain records */
    float log_evalue_threshold;
    float search_space;       /* effective search space (bit scores) */
} cbp_hits_input;
int cbp_format_hits_host(const cbp_hits_input* in, const cbp_format_options* fo, char* buf,
                         size_t cap, size_t* used, size_t* nhits);

/* Merge the sorted hit lists of a query's database chunks (parts) by log
 * E-value, stably (equal values keep part order, then list order), as the
 * reference's writer joins them. log_evalues[p][i] is the log E-value of
 * hit i of part p. Writes part[] and index[] (sum of counts entries each;
 * either may be NULL). */
int cbp_merge_hit_lists(size_t nparts, const float* const* log_evalues, const size_t* counts,
                        int32_t* part, int32_t* index);

/* What the report says besides the hits. */
typedef struct cbp_report_info {
    const char* program;              /* program name (NULL: none) */
    const char* version;              /* version (NULL: none) */
    const char* const* references;    /* NULL-terminated list of citation lines, or NULL */
    int query_len;
    const char* query_desc;           /* query description (NULL: none) */
    const char* const* db_names;      /* database names */
    size_t n_db_names;
    uint64_t db_size;                 /* total database positions */
    uint64_t db_entries;              /* database profiles */
    float log_evalue_threshold;
    float search_space;               /* effective search space */
    int delta_length;                 /* length adjustment */
    float ref_lambda, ref_k;          /* ungapped reference values */
    float gapped_lambda, gapped_k;    /* gapped values */
    int nohits;                       /* NOHITS: annotations listed */
    int noalns;                       /* NOALNS: hit records listed */
} cbp_report_info;

/* The per-query report text from the merged hits (annotations[i],
 * hit_records[i] in final order, as cbp_format_hits gives them). With buf ==
 * NULL only *used is set; a smaller buffer gives CBP_ERR_LIMIT. */
int cbp_write_report(const cbp_report_info* info, const cbp_format_options* fo,
                     const char* const* annotations, const char* const* hit_records, size_t nhits,
                     char* buf, size_t cap, size_t* used);

/* Karlin-Altschul parameters of the statistical configuration (cother.par:
 * [UNGAPPED] lambda, K; [GAPPED_A_1] lambda, K, alpha, beta). Defaults are
 * the reference's shipped values. */
int cbp_set_karlin_altschul(cbp_context* ctx, float ungapped_lambda, float ungapped_k,
                            float gapped_lambda, float gapped_k, float gapped_alpha,
                            float gapped_beta);

/* ------------------------------------------------------------------------
 * Allocation-free phase-1 DP. This entry point has no counterpart in the
 * reference.
 *
 * For callers that cannot allocate device memory when they run the search
 * (their device memory belongs to their own pool allocator, or a cudaMalloc
 * would synchronise the device where they enqueue work). The caller owns
 * every input and output as device memory; the only scratch of the DP --
 * the strip that carries each band's bottom row to the next band -- is a
 * fixed array inside the library of 5 * CBP_NOALLOC_MAX_COLUMNS floats
 * (1.25 MiB), which every GPU that loads the library keeps until the process
 * exits. The call allocates and frees nothing.
 *
 * Inputs (device pointers, the layout of the other entry points):
 *   scores     [query_len][ld] slab score matrix (column c = chunk position
 *              first_column + c); ld <= CBP_NOALLOC_MAX_COLUMNS, else
 *              CBP_ERR_LIMIT;
 *   query_trn  [7][query_len+1] query transitions (entry r = into position r);
 *   db_trn     [7][db_npos+db_nprof] chunk transitions, the beginning
 *              vector of profile p at entry prof_start[p]+p;
 *   prof_len, prof_start  [db_nprof] lengths and first positions;
 *   profiles first_profile .. first_profile+nprof-1 are processed.
 * Preconditions on every processed profile p (device data, so they are
 * checked by the kernel, not before the launch): its columns lie inside the
 * slab, 0 <= prof_start[p] - first_column and
 * prof_start[p] - first_column + prof_len[p] <= ld, and prof_len[p] < 65536
 * (cell coordinates are packed into 16 + 16 bits; query_len < 65536 is
 * checked before the launch, CBP_ERR_LIMIT). A profile that breaks either is
 * skipped: nothing of it is read or written, its max_scores entry is NaN and
 * its max_coords entry 0xffffffff.
 * Outputs (device): btck [query_len][ld] backtrack codes, max_scores and
 * max_coords [nprof] (maximum MM score and its cell (x<<16)|y).
 * The work is enqueued on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and the call returns after the launch.
 *
 * Every call looks up the scratch array's device address
 * (cudaGetSymbolAddress) with the caller's device current, so a device reset
 * between calls is safe. The first lookup on a device loads the library's
 * device code there: make that first call before any stream capture. All
 * calls share the one scratch array and it
 * keeps the last call's contents (the DP needs no zeroed scratch: the first
 * band never reads the strip); calls whose work overlaps on the GPU race on
 * it and must be serialised by the caller, e.g. on one stream. */
#define CBP_NOALLOC_MAX_COLUMNS 65536
int cbp_dp1_noalloc(const float* scores, size_t ld, int query_len, const float* query_trn,
                    long long db_npos, int db_nprof, const float* db_trn,
                    const int* prof_len, const long long* prof_start,
                    int first_profile, int nprof, long long first_column,
                    uint8_t* btck, float* max_scores, uint32_t* max_coords,
                    void* stream);

/* ------------------------------------------------------------------------
 * Request loop over a resident database (serving). No counterpart in the
 * reference, which is a batch program: its job dispatcher hands whole
 * queries to per-GPU workers (src/libmycu/cualn/JobDispatcher.cpp:1124-1133),
 * each searching one query at a time (DevCommThread.cpp:316-355).
 *
 * A server keeps one database chunk resident on a GPU and searches queries
 * as they arrive, through `slots` contexts sharing the chunk (each with its
 * own stream, working memory and worker thread). When a slot is free the
 * oldest waiting query and the ones behind it, up to `max_batch`, are
 * searched together in one pass over the database (cbp_process_batch), as
 * long as the stacked queries' slab still holds the longest profile. A
 * batch is charged the device memory of one slab of its stacked rows
 * (cbp_slab_bytes), the slab cut so that a batch takes at most `max_share`
 * of the budget; batches are admitted in arrival order while the charges
 * of all slots (each slot's largest so far) stay within the budget. */
typedef struct cbp_server cbp_server;

typedef struct cbp_server_config {
    int device;             /* GPU */
    int slots;              /* concurrent batches (contexts), 1..64 */
    int max_batch;          /* queries searched in one pass at most */
    size_t budget_bytes;    /* device memory for the slots' working buffers
                             * (0 = 70 % of the free memory after the upload) */
    double max_share;       /* largest share of the budget one batch may take */
    uint64_t db_len;        /* database totals for E-values (0 = the chunk's) */
    size_t n_seqs;
} cbp_server_config;

/* Times (seconds of a steady clock) and shape of a finished request. */
typedef struct cbp_server_result {
    double arrival_s, start_s, finish_s;
    int slot, batch;                 /* the slot that searched it, queries in its batch */
    size_t slab_positions;           /* slab size the batch was searched with */
    size_t nrecords, nhits, alignment_length;
} cbp_server_result;

/* The admission rule (host only, no device): for a batch needing `need`
 * bytes, the free slot (busy[i] == 0) whose growth of its charge held[i]
 * keeps the sum within `budget`, the least growth first, with
 * *grant = need; -1 (wait) while a busy slot would have room once done;
 * else the free slot with the most room, if that is at least min_grant,
 * with *grant = its room (the batch then runs with a smaller slab). */
int cbp_ledger_choose(const size_t* held, const char* busy, size_t nslots, size_t budget, size_t need,
                      size_t min_grant, size_t* grant);

/* slots 3, max_batch 4, budget 0 (auto), max_share 0.5, totals 0 */
void cbp_server_default_config(cbp_server_config* cfg);
/* Upload the chunk (the 181 field pointer tables, as cbp_transfer_chunk
 * takes them) and start the server's threads. */
int cbp_server_create(const cbp_server_config* cfg, const cbp_options* opt, const float* ss_table,
                      char* const* db_pmbeg, char* const* db_pmend, cbp_server** server);
/* The memory budget the server admits batches against. */
int cbp_server_budget(cbp_server* server, size_t* budget_bytes);
/* Queue a query (its field tables are copied; the caller may free them on
 * return); *ticket identifies the request. CBP_ERR_MEMORY when the budget
 * cannot hold a slab of the longest profile for this query. */
int cbp_server_submit(cbp_server* server, size_t query_len, char* const* qpmbeg, char* const* qpmend,
                      uint64_t* ticket);
/* Wait for a request (timeout_ms < 0: without limit; CBP_ERR_STATE when it
 * is not done in time); *info (may be NULL) receives its times and sizes.
 * Returns the search's status. */
int cbp_server_wait(cbp_server* server, uint64_t ticket, int timeout_ms, cbp_server_result* info);
/* A finished request's results: hit records (CBP_REC_FLOATS each), the
 * first max_hits of its hit order, the 5 alignment rows (row_stride >= the
 * alignment length). Any output may be NULL. */
int cbp_server_get(cbp_server* server, uint64_t ticket, float* records, size_t max_records,
                   int32_t* order, size_t max_hits, char* rows, size_t row_stride);
/* Forget a finished request's results. */
int cbp_server_release(cbp_server* server, uint64_t ticket);
/* Finish the queued requests, stop the threads, free everything. */
int cbp_server_destroy(cbp_server* server);
/* Message of the last failed server call on the calling thread. */
const char* cbp_server_last_error(void);

/* Limit the number of database positions processed per slab (0 = plan by
 * the memory budget). Used to exercise multi-slab processing. */
int cbp_set_max_slab_positions(cbp_context* ctx, size_t max_positions);

/* The kernel variants in use for queries of length query_len (the tuner's
 * choice for its bin, or the defaults 16 / 1024 / 2 before tuning or with
 * autotune = 0): score-kernel query rows per block, column-ordering window,
 * phase-1 DP warps per block; and in ms[0..n) the tuned candidates' times on
 * the sample (score variants (16,1024), (8,1024), (32,1024), (16,256),
 * (16,4096), then DP variants 2 and 1 warps). */
int cbp_get_tuning(cbp_context* ctx, size_t query_len, int* rows, int* window, int* dp_warps,
                   float* ms, int n);

/* Fix the kernel variants for queries in query_len's bin (no tuning
 * there): rows 8/16/32, window a multiple of 32 up to 4096, dp_warps 1/2. */
int cbp_set_kernels(cbp_context* ctx, size_t query_len, int rows, int window, int dp_warps);

/* Device time in milliseconds of the kernels of the last cbp_process()
 * call, per stage: [0] score matrix, [1] phase-1 DP, [2] phase-1
 * finalization, [3] statistics, [4] MAP phase, [5] result assembly.
 * Returns the number of stages written (<= n). */
int cbp_stage_times(cbp_context* ctx, float* ms, int n);

/* Kernel launches of the last cbp_process() call per stage (same stage
 * order as cbp_stage_times). Returns the number of stages written. */
int cbp_stage_launches(cbp_context* ctx, uint64_t* launches, int n);

/* Number of CUDA-graph launches since the context was created: with the
 * plain form each slab's phase 1 (column order, score matrix, DP,
 * finalization, pass list) runs as one executable graph, captured on the
 * slab's parameters and updated in place (no counterpart in the
 * reference, which launches once per block diagonal from the host). */
int cbp_graph_launches(cbp_context* ctx, uint64_t* graphs);

/* Number of kernel launches issued by the last cbp_process() call. */
int cbp_launch_count(cbp_context* ctx, uint64_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* COTHER_B200_H */
