/*
 * msg_b200.h -- C ABI of the B200 (sm_100a) read-mapping library that stands
 * in for MSGseqTK's seeding -> locate -> chaining -> DP path, with the host
 * pieces around it (database files, FASTQ in, the likelihood/MAPQ/pairing
 * tail, SAM text out) and msgseqtk-clean's MEM log-odds path.
 *
 * The reference has no FFI; its "operator API" is a set of C++ classes called
 * from the per-read task bodies of msgseqtk-align (src/msgseqtk-align.cpp:610-628
 * for single-end, :680-705 for each mate of a pair). Each entry point below
 * names the reference interface it replaces. Plain pointers and sizes only;
 * all host buffers belong to the caller; no exceptions cross the ABI; every
 * function returns an msg_status.
 *
 * Threading: one host thread per msg_ctx (calls on one context are not
 * re-entrant); contexts are independent. Each context owns one CUDA stream.
 * A call on a context runs on the context's device and gives the calling
 * thread's current device back before it returns.
 *
 * Devices: the library carries sm_100a (B200) code only; msg_ctx_create
 * returns MSG_EUNSUPPORTED on any other architecture.
 */
#ifndef MSG_B200_H
#define MSG_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum msg_status {
    MSG_OK = 0,
    MSG_EINVAL = 1,        /* bad argument (null pointer, inconsistent sizes) */
    MSG_ENOMEM = 2,        /* device or host allocation failed */
    MSG_EUNSUPPORTED = 3,  /* input the CUDA path does not implement (see msg_strerror) */
    MSG_ETIMEOUT = 4,      /* a bounded device wait ran out */
    MSG_ECUDA = 5,         /* CUDA runtime error */
    MSG_ESTATE = 6,        /* call out of order (e.g. mapping before an index is loaded) */
    MSG_EINTERNAL = 7      /* a device-side consistency check failed */
} msg_status;

/* Human-readable text for a status code (static storage). */
const char* msg_strerror(int status);

typedef struct msg_ctx msg_ctx;

/* Detail of the last failure on this context (valid until the next call). */
const char* msg_last_error(const msg_ctx* ctx);

/* Create a context on CUDA device `device`. */
int msg_ctx_create(int device, msg_ctx** out);
void msg_ctx_destroy(msg_ctx* ctx);

/* Decoded FMD-index, as FMDIndex holds it (src/FMDIndex.h:337-343):
 * the BWT as nt16 codes (getBWT, FMDIndex.cpp:195), base counts B[0..15]
 * (C[] is derived exactly as buildCounts does, FMDIndex.cpp:118-129), and the
 * SA sample set -- rows flagged in SAidx (i % 32 == 0 or BWT[i] == 0,
 * FMDIndex.cpp:465-480) with their SAsampled values, rows ascending. */
typedef struct msg_fmd_view {
    int64_t n;
    const uint8_t* bwt;
    const int64_t* base_count;   /* 16 entries */
    int64_t n_samples;
    const int64_t* sample_rows;
    const int64_t* sample_vals;
} msg_fmd_view;

/* MetaGenome coordinate table and target sequences (src/MetaGenome.h:147-167,
 * 237-261, 319-321): per chromosome (tid order) its BD start/end, its length
 * WITHOUT the terminator, and the forward nt16 sequences concatenated at
 * chr_off[t] .. chr_off[t+1]. */
typedef struct msg_mtg_view {
    int64_t n_chrom;
    const int64_t* bd_start;
    const int64_t* bd_end;
    const int64_t* chr_len;
    const uint8_t* chr_seq;
    const int64_t* chr_off;      /* n_chrom + 1 entries */
} msg_mtg_view;

/* Load an index into device memory (replaces FMDIndex::load + MetaGenome::load
 * for the mapping path, src/msgseqtk-align.cpp:444-508). Builds the device
 * image: 2-bit BWT with occurrence buckets, the full suffix array (recovered
 * on the device from the SA samples), and the chromosome table. */
int msg_index_load(msg_ctx* ctx, const msg_fmd_view* fmd, const msg_mtg_view* mtg);

/* ---- Database files ----
 * Read a database as msgseqtk-build writes it (src/msgseqtk-build.cpp:382-426):
 * the MetaGenome (.mtg, MetaGenome::save), its sequences (.mgs,
 * MetaGenome::saveSeq) and the FMD-index (.fmd, FMDIndex::save, whose BWT is
 * an RRR-compressed wavelet tree). The BWT is decoded on n_threads host
 * threads. Replaces MetaGenome::load/loadSeq + FMDIndex::load
 * (src/msgseqtk-align.cpp:444-508) for callers without the reference's
 * libraries. msg_db_views then gives the views msg_index_load takes (valid
 * until msg_db_free). MSG_EINVAL for unreadable or inconsistent files. */
typedef struct msg_db msg_db;
int msg_db_read(const char* mtg_path, const char* mgs_path, const char* fmd_path, int n_threads, msg_db** db);
int msg_db_views(const msg_db* db, msg_fmd_view* fmd, msg_mtg_view* mtg);
void msg_db_free(msg_db* db);

/* msg_db_read with the BWT decoded on the GPU `device`: the same database,
 * the same checks (MSG_EINVAL for files msg_db_read rejects), the RRR bit
 * sequences unranked, the wavelet tree walked (WaveletTreeRRR::access,
 * src/libsds/src/WaveletTreeRRR.cpp:58-76) and the sampled rows listed by
 * device kernels instead of host threads. Device memory is held only during
 * the call (about 2.5 bytes per BD symbol); the result lives on the host. */
int msg_db_read_device(int device, const char* mtg_path, const char* mgs_path, const char* fmd_path, msg_db** db);

/* msg_db_read with a decoded image of the database kept at image_path (e.g.
 * "<db>.fmd.b200"), the load step of the same call sites. The image holds the
 * decoded arrays and is keyed by the sizes and 64-bit content hashes of the
 * three files: when the key and the image's own body hash match, the database
 * is read from it (no wavelet-tree decode; *from_image = 1); otherwise the
 * files are decoded and the image is written anew next to its path and
 * renamed into place (*from_image = 0, or -1 when it could not be written,
 * which is not an error). from_image may be NULL. */
int msg_db_read_cached(const char* mtg_path, const char* mgs_path, const char* fmd_path, const char* image_path,
                       int n_threads, msg_db** db, int* from_image);

/* Device bytes held by the loaded index. */
int msg_index_bytes(const msg_ctx* ctx, int64_t* bytes);

/* Let `ctx` map against the index `owner` loaded, without a second copy in
 * device memory (both contexts on the same device). The reference's mapping
 * tasks share one read-only FMDIndex and MetaGenome across OpenMP threads
 * (src/msgseqtk-align.cpp:600-607, the const pointers held at SMEM.h:192-194
 * and Alignment.h:352-355); this is the same sharing across contexts, so that
 * several host threads, one context each, can map batches side by side on
 * their own streams. The index memory lives until the last context holding
 * it is destroyed or loads another index; reloading `owner` afterwards does
 * not change what `ctx` maps against. Kernel shapes and the band model are
 * per context and are not copied. Waits for `ctx`'s own stream first.
 * MSG_ESTATE if `owner` has no index. */
int msg_ctx_share_index(msg_ctx* ctx, const msg_ctx* owner);

/* Mapping parameters (src/msgseqtk-align.cpp:183-397 defaults). */
typedef struct msg_map_params {
    int64_t min_len;        /* --min-seed, SMEM::MIN_LENGTH = 17 */
    double max_evalue;      /* --max-evalue, SMEM::MAX_EVALUE = 0.01; +inf for no limit */
    int64_t max_nseed;      /* --max-nseed, SMEM::MAX_NSEED = 500 */
    int32_t mode;           /* 0 = GLOBAL (NW, default), 1 = LOCAL (SW) */
    /* ScoreScheme (src/ScoreScheme.cpp:14-18); integral values only */
    double match, mismatch, gap_open, gap_ext;
    /* Alignment::filter (src/Alignment.cpp:548-555; --min-score, default
     * 0.65 in msgseqtk-align): records with alnScore < read length *
     * min_score_rate are removed on the device, as the reference does right
     * after buildAlignments (src/msgseqtk-align.cpp:628, 704-705). A negative
     * value (the default here) keeps every record buildAlignments makes. */
    double min_score_rate;
    /* DP cells of the 5' and 3' flank rectangles (GLOBAL mode only):
     * 0 = the reference's whole rectangles (default); 1 = a diagonal band of
     * half-width band_w (0..31) around the adjacent seed's diagonal; 2 = a band width
     * chosen per chain by the model loaded with msg_band_model_set. A banded
     * chain is kept only under a score-bound certificate: either no path
     * through a cell outside the band can reach the banded score (the record
     * is then the reference's), or no path at all can reach the filter's
     * threshold (the reference would filter the record; needs
     * min_score_rate >= 0). Any other chain is recomputed on the whole cell
     * set, so the records never depend on the band. */
    int32_t band_mode;
    int32_t band_w;
} msg_map_params;

/* Fill defaults. */
void msg_map_params_default(msg_map_params* p);

/* A batch of reads: nt16 codes concatenated, read i at seq[off[i] .. off[i+1]). */
typedef struct msg_read_batch {
    int64_t n_reads;
    const uint8_t* seq;
    const int64_t* off;     /* n_reads + 1 entries */
} msg_read_batch;

/* One alignment per seed chain, in the order Alignment::buildAlignments
 * produces them (src/Alignment.cpp:420-427), before Alignment::filter.
 * Coordinates follow Alignment's fields (src/Alignment.h:357-372). */
typedef struct msg_aln {
    int64_t read;           /* index of the read in the batch */
    int32_t tid;
    int32_t strand;         /* GLoc::STRAND: 1 = FWD, 2 = REV */
    int64_t t_start, t_end; /* DP window on the chromosome */
    int64_t aln_from, aln_to, aln_start, aln_end;
    int32_t aln_score;      /* integral; the reference stores it as a double */
    int32_t flags;          /* bit0: last row held no finite score; bit1: traceback left the matrix */
    int64_t cigar_off;      /* CIGAR words (SAM encoding len<<4|op) in the output's cigar array */
    int32_t n_cigar;
    int32_t pad;
} msg_aln;

/* Output buffers owned by the caller. The library fills at most *_cap entries
 * and always reports the counts it needed in n_aln / n_cigar; when a count
 * exceeds its capacity the call returns MSG_EINVAL with nothing else valid.
 * When aln, cigar and read_aln_off are all NULL the results stay in the
 * context's device buffers (see msg_result_device) and only the counts are
 * returned. */
typedef struct msg_aln_out {
    int64_t aln_cap;
    msg_aln* aln;
    int64_t cigar_cap;
    uint32_t* cigar;
    int64_t n_aln;          /* out */
    int64_t n_cigar;        /* out */
    int64_t* read_aln_off;  /* optional, n_reads + 1: alignments of read i are aln[off[i] .. off[i+1]) */
} msg_aln_out;

/* Optional per-stage dumps for parity checks (any pointer may be NULL). */
typedef struct msg_stage_dump {
    /* SMEMs in SMEM_LIST::findAllSMEMS emission order (src/SMEM.cpp:186-215),
     * rows of 6 int64: from, to, fwdStart, revStart, size, logP bit pattern */
    int64_t smem_cap;
    int64_t* smem;
    int64_t* smem_off;      /* n_reads + 1 */
    /* seeds after SeedPair::removeRedundant (src/SeedPair.cpp:71-88), rows of
     * 6 int64: from, to, start, end, tid, strand */
    int64_t seed_cap;
    int64_t* seed;
    int64_t* seed_off;      /* n_reads + 1 */
    int64_t n_smem, n_seed; /* out */
} msg_stage_dump;

/* Statistics of the last mapping call. */
typedef struct msg_map_stats {
    int64_t n_reads, n_smem, n_seed, n_chain, n_aln;
    int64_t n_ext;          /* bi-interval extensions that reached the occurrence lookup */
    int64_t n_sa;           /* suffix-array rows located */
    int64_t dp_cells;       /* cells of the reference DP cell set (rectangles + seed diagonals) */
    int64_t host_sorted;    /* reads whose SMEM order needed the host std::sort */
    int64_t n_launch;       /* kernels of this library launched by the call */
    double ms_total, ms_smem, ms_locate, ms_chain, ms_dp;
    int64_t dp_cells_done;  /* DP cells actually computed (bands, whole rectangles, recomputations) */
    int64_t n_band_exact;   /* banded chains certified identical to the reference */
    int64_t n_band_drop;    /* banded chains certified below the filter threshold */
    int64_t n_band_fallback;/* banded chains recomputed on the whole cell set */
    int64_t n_filtered;     /* records removed by min_score_rate (drops included) */
    int64_t n_dp_warp;      /* chains whose DP ran one warp each (the rest: one thread each) */
    int64_t n_dp_class[5];  /* chains per DP class: row by row, stripes, banded stripes, warp, banded warp */
    int64_t dp_class_cells[5]; /* cells computed per class (recomputations count with the warp class) */
    int64_t n_smem_rerun;   /* reads the one-thread SMEM kernel gave to the warp kernel (candidate list too long) */
    int64_t smem_retries;   /* SMEM stage reruns with larger output slots */
    int64_t n_ext_ff;       /* bi-interval extensions of unique matches done by text comparison instead */
    int64_t n_ff_steps;     /* steps of those comparisons (a suffix-array word, a 16-byte text chunk or an
                               inverse-suffix-array word loaded each) */
    double ms_dp_part[4];   /* ms_dp by part: chain preparation and storage sizing, band classes and sort,
                               fills and tracebacks, filter and CIGARs */
} msg_map_stats;

/* Map a batch of reads held in HOST memory: the per-read SE task body
 * findSeeds -> getChains -> buildAlignments (src/msgseqtk-align.cpp:612-625;
 * SMEM_LIST::findSeeds src/SMEM.cpp:271, SeedChain::getChains
 * src/SeedChain.cpp:40, Alignment::buildAlignments src/Alignment.cpp:420).
 * For paired-end data call it on both mates (findSeedsPE, src/SMEM.h:383-389,
 * is two independent findSeeds calls). `dump` may be NULL. */
int msg_map_batch(msg_ctx* ctx, const msg_read_batch* reads, const msg_map_params* params,
                  msg_aln_out* out, msg_stage_dump* dump);

/* msg_map_batch over n_batches batches in HOST memory, with the copies
 * overlapped: batch k+1's reads go to the device on a second stream while
 * batch k is mapped, and batch k's records come back while batch k+1 is
 * mapped (pin the host buffers for the copies to overlap). outs[k] receives
 * batch k's results exactly as msg_map_batch would (every output pointer
 * required except read_aln_off). When a batch's counts exceed its capacities
 * the call still maps the others and returns MSG_EINVAL with those counts in
 * outs[k]. No reference counterpart (a batching form of msg_map_batch). */
int msg_map_batches(msg_ctx* ctx, int64_t n_batches, const msg_read_batch* reads, const msg_map_params* params,
                    msg_aln_out* outs);

/* ---- The mapping task one stage at a time ----
 * msg_map_batch runs these stages fused on the device; each call below stops
 * at one of the reference's own operator boundaries and takes and returns
 * host arrays, so a caller can inspect or replace any step (reads in host
 * memory as for msg_map_batch; results identical to the fused call's).
 * Caller arrays are checked before any kernel reads them (MSG_EINVAL). */

/* SMEM_LIST::findAllSMEMS (src/SMEM.cpp:186-215), the first step of
 * SMEM_LIST::findSeeds (src/SMEM.cpp:272): per read its SMEMs in emission
 * order as rows of 6 int64 (from, to, fwdStart, revStart, size, logP bit
 * pattern; the SMEM fields of src/SMEM.h:196-200), read i's at rows
 * smem_off[i] .. smem_off[i+1) (n_reads + 1 offsets). *n_smem receives the
 * row count; MSG_EINVAL, rows not written, when it exceeds smem_cap. */
int msg_seed_batch(msg_ctx* ctx, const msg_read_batch* reads, const msg_map_params* params, int64_t* smem,
                   int64_t smem_cap, int64_t* smem_off, int64_t* n_smem);

/* SMEM::getSeeds (src/SMEM.cpp:244-269, with FMDIndex::accessSA and
 * MetaGenome::getTid/getLoc/getStrand) of the SMEM rows the caller keeps
 * after findSeeds' sort and maxNSeed cut (src/SMEM.cpp:275-300; read i's
 * rows at smem_off[i] .. smem_off[i+1)), then SeedPair::removeRedundant
 * (src/SeedPair.cpp:71-88): per read its seeds as rows of 6 int64 (from, to,
 * start, end, tid, strand: SeedPair's fields) in the order removeRedundant
 * leaves them, read i's at seed_off[i] .. seed_off[i+1). *n_seed receives
 * the count; MSG_EINVAL, rows not valid, when it exceeds seed_cap. An SMEM
 * row must lie in its read (0 <= from < to <= length) and address
 * suffix-array rows of the index (fwdStart, revStart >= 0, + size <= n). */
int msg_locate_batch(msg_ctx* ctx, const msg_read_batch* reads, const int64_t* smem, const int64_t* smem_off,
                     int64_t* seed, int64_t seed_cap, int64_t* seed_off, int64_t* n_seed);

/* SeedChain::getChains (src/SeedChain.cpp:40-73; maxMismatch = ceil(L*0.2)
 * and maxIndel = ceil(L*0.1) as msgseqtk-align sets them,
 * src/msgseqtk-align.cpp:619-620) on each read's seeds (rows as
 * msg_locate_batch returns them): chain k of the batch holds the seeds
 * chain_seed[chain_seed_off[k] .. chain_seed_off[k+1]), indices into its
 * read's seed rows; read i's chains are read_chain_off[i] ..
 * read_chain_off[i+1). *n_chain and *n_chain_seed receive the counts;
 * MSG_EINVAL when they exceed chain_cap (chain_seed_off holds chain_cap + 1
 * entries) or chain_seed_cap. Seeds must lie in their read and chromosome
 * (end - start == to - from, tid < chromosomes, strand 1 or 2). */
int msg_chain_batch(msg_ctx* ctx, const msg_read_batch* reads, const int64_t* seed, const int64_t* seed_off,
                    int32_t* chain_seed, int64_t chain_seed_cap, int64_t* chain_seed_off, int64_t chain_cap,
                    int64_t* read_chain_off, int64_t* n_chain, int64_t* n_chain_seed);

/* Alignment::buildAlignments (src/Alignment.cpp:420-427: the window,
 * calculateScores, backTrace and getAlnCigar of each chain) for chains as
 * msg_chain_batch returns them: one record per chain in chain order,
 * exactly as msg_map_batch returns them (params: mode, score scheme,
 * min_score_rate, band_mode/band_w; the seeding fields are not used). A
 * chain's seeds must ascend in the read's list, not overlap in the read or
 * the target, and share tid and strand. */
int msg_align_batch(msg_ctx* ctx, const msg_read_batch* reads, const int64_t* seed, const int64_t* seed_off,
                    const int32_t* chain_seed, const int64_t* chain_seed_off, const int64_t* read_chain_off,
                    const msg_map_params* params, msg_aln_out* out);

/* Same as msg_map_batch with the reads already in device memory (seq and off
 * are device pointers); results still land in the caller's host buffers. */
int msg_map_batch_device(msg_ctx* ctx, const msg_read_batch* dev_reads, const msg_map_params* params,
                         msg_aln_out* out, msg_stage_dump* dump);

int msg_last_stats(const msg_ctx* ctx, msg_map_stats* stats);

/* Device pointers to the last call's results (valid until the next mapping
 * call on this context): msg_aln records, CIGAR words, per-read offsets. */
int msg_result_device(const msg_ctx* ctx, const msg_aln** aln, const uint32_t** cigar, const int64_t** read_aln_off);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or events against the library's. */
int msg_ctx_stream(const msg_ctx* ctx, void** stream);

/* Bound the device memory the DP uses for its rectangle storage (default
 * 16 GiB). No reference counterpart (the reference allocates three
 * (L+1) x (T+1) double matrices per chain). A batch whose chains need more
 * (long reads with large flanks) is aligned over consecutive ranges of
 * chains that fit; a single larger chain gets a range of its own. Results do
 * not depend on the limit. */
int msg_ctx_set_scratch_limit(msg_ctx* ctx, int64_t bytes);

/* Work split of the DP stage. No reference counterpart (the reference fills
 * every chain's matrices on one CPU thread). Unbanded chains of at most
 * small_area rectangle cells are filled row by row by one GPU thread; chains
 * of at most warp_area cells by one thread in register stripes of
 * stripe_rows rows (8, 16 or 32); larger chains by a warp along
 * anti-diagonals. Defaults 64, 262144, 16. Results do not depend on it. */
int msg_ctx_set_dp_shape(msg_ctx* ctx, int32_t stripe_rows, int64_t small_area, int64_t warp_area);

/* Lane width of the register-stripe DP fill (no reference counterpart):
 * 16 (default) = unbanded chains in GLOBAL mode whose every finite value lies
 * within +-8191 by a score bound ((L + T + 1) * max(match, mismatch,
 * gap_open + gap_ext) < 8192) run two 16-row stripes per thread in 16-bit
 * halves of each register, two cells per DP instruction; 32 = every chain
 * in 32-bit values. Results do not depend on it. */
int msg_ctx_set_dp_lanes(msg_ctx* ctx, int32_t bits);

/* Register budget of the register-stripe DP kernel (no reference
 * counterpart): sized for 3 (default; 168 registers, no spills in the
 * 16-bit fill) or 4 (128 registers, more warps) resident blocks of 128
 * threads per SM. Results do not depend on it. */
int msg_ctx_set_dp_occupancy(msg_ctx* ctx, int32_t blocks);

/* Kernel shape of the SMEM stage for reads up to 254 bp (no reference
 * counterpart): 0 = one read per thread (default); 1 and 2 = two reads per
 * thread, each thread keeping two extensions' bucket loads in flight (1:
 * registers sized for 4 blocks of 128 threads per SM, 2: for 3); 3 and 4 =
 * one read per thread, the candidates of one pass of findFwdBackSMEMS /
 * findBackFwdSMEMS (SMEM.cpp:93-116, 148-171) extended up to 4 (3) or 2 (4)
 * at a time, their bucket loads in flight together; 5 and 6 = variant 0 with
 * registers sized for 6 and 8 resident blocks of 128 threads per SM (more
 * warps, some spilling) instead of 5; 7 = variant 0 with the fast-forward
 * over unique matches (a run of extensions of a size-1 interval -- a
 * walk's, or a pass's single candidate's -- replaced by comparing the read
 * with the BD text before the match's suffix-array position and one
 * inverse-suffix-array lookup). Results do not depend on it. */
int msg_ctx_set_smem_shape(msg_ctx* ctx, int32_t variant);

/* The shapes chosen by msg_autotune, with the stage times that chose them. */
typedef struct msg_tune {
    int32_t stripe_rows;
    int32_t n_tried;        /* shapes timed */
    int64_t small_area, warp_area;
    double ms_dp;           /* DP stage time of the chosen split on the sample */
    double ms_dp_default;   /* the same with the defaults (16, 64, 262144) */
    int32_t smem_variant;
    int32_t dp_lanes;       /* 16 or 32 (msg_ctx_set_dp_lanes) */
    double ms_smem;         /* SMEM stage time of the chosen variant */
    double ms_smem_default; /* the same with variant 0 */
    int32_t dp_stripe_blocks; /* 3 or 4 (msg_ctx_set_dp_occupancy) */
    int32_t pad2;
} msg_tune;

/* Autotuner of the kernel shapes (no reference counterpart): maps the sample
 * batch (host memory) with `params` under candidate shapes -- the SMEM
 * variant, then the DP warp threshold, stripe height, row-by-row threshold,
 * lane width and stripe-kernel register budget, each chosen with the others
 * fixed -- timing the stage it
 * affects (a second run of every shape, after one untimed), and sets the
 * fastest on the context. Records never depend on the shapes, so the choice
 * only changes speed. */
int msg_autotune(msg_ctx* ctx, const msg_read_batch* sample, const msg_map_params* params, msg_tune* result);

/* ---- Seeding that allocates nothing ----
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc/cudaFree while mapping -- a host application whose GPU memory is
 * all owned by its own allocator (a framework's caching pool, or a fixed
 * reservation carved out at start-up), where an extra device allocation would
 * fail or fragment that budget. It runs the same SMEM search as msg_map_batch
 * (SMEM_LIST::findAllSMEMS per read, src/SMEM.cpp:186-215) with every input
 * and output in caller-owned DEVICE memory: reads (d_seq, d_off as in
 * msg_read_batch), SMEM rows (6 int64 each, as in msg_stage_dump) written to
 * d_smem at row r * cap_per_read for read r, and per-read counts in d_count.
 * Its working memory is one static device array of fixed size that every GPU
 * loading this library holds until exit (about 14 MB with the limits below);
 * reads longer than MSG_NOALLOC_MAX_READ_LEN are rejected with MSG_EINVAL.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) and caches it; make that first call before any
 * stream capture on the device. All calls share the array: calls that overlap
 * on the GPU (two contexts or threads at once) race and must be serialised by
 * the caller. A count above cap_per_read returns MSG_EINVAL with the needed
 * counts left in d_count. */
#define MSG_NOALLOC_MAX_READ_LEN 320
#define MSG_NOALLOC_WARPS 1184
int msg_smem_batch_noalloc(msg_ctx* ctx, int64_t n_reads, const uint8_t* d_seq, const int64_t* d_off,
                           const msg_map_params* params, int64_t* d_smem, int64_t cap_per_read, int32_t* d_count);

/* ---- Learned band model ----
 * No counterpart in the reference (its DP always uses the whole rectangles).
 * The model is a 16 -> 64 -> 64 -> 4 ReLU network over chain statistics whose
 * classes are band half-widths 7, 15, 31 and "whole rectangle". Parameters
 * are MSG_BAND_NPARAMS floats: feature mean[16], feature scale[16], W1[64][16],
 * b1[64], W2[64][64], b2[64], W3[4][64], b3[4]; weights are used in bf16 with
 * fp32 accumulation. */
#define MSG_BAND_FEATURES 16
#define MSG_BAND_HIDDEN 64
#define MSG_BAND_CLASSES 4
#define MSG_BAND_NPARAMS 5540

/* Load parameters (host floats) for band_mode 2. */
int msg_band_model_set(msg_ctx* ctx, const float* params, int64_t n_params);

/* Training data from a batch: per chain (in record order of msg_map_batch),
 * MSG_BAND_FEATURES features and the label = the class whose DP costs the
 * fewest cells once certified (an uncertified band costs its cells plus the
 * whole rectangles; ties go to the wider class), with the certificate of
 * `params` (min_score_rate included); -1 for chains that never get a band
 * (small chains, flanks that a band would not cut). Host buffers of cap
 * chains; *n_chain receives the chain count (MSG_EINVAL when it exceeds cap). */
int msg_band_collect(msg_ctx* ctx, const msg_read_batch* reads, const msg_map_params* params, float* feat,
                     int32_t* label, int64_t cap, int64_t* n_chain);

typedef struct msg_band_train_params {
    int32_t epochs;
    int32_t batch;          /* samples per Adam step */
    float lr;               /* Adam step size (beta1 0.9, beta2 0.999, eps 1e-8) */
    uint64_t seed;          /* initialisation and shuffling */
} msg_band_train_params;

/* Train the model on the GPU (host features and labels of n samples).
 * params receives the trained parameters (feature mean/scale from the data);
 * loss (epochs floats, may be NULL) the mean cross entropy of each epoch.
 * The context's model is set to the result. */
int msg_band_train(msg_ctx* ctx, const float* feat, const int32_t* label, int64_t n,
                   const msg_band_train_params* tp, float* params, float* loss);

/* Gradient of the mean cross entropy over n samples at `params` (the first
 * 2*MSG_BAND_FEATURES entries, mean and scale, are not trained): grad
 * receives MSG_BAND_NPARAMS - 2*MSG_BAND_FEATURES floats in the parameter
 * order, *loss the mean loss. For checking the training kernels. */
int msg_band_grad(msg_ctx* ctx, const float* params, const float* feat, const int32_t* label, int64_t n,
                  float* grad, float* loss);

/* ---- Host tail of the single-end task (runs on host threads, no GPU) ---- */

typedef struct msg_tail_params {
    double min_score_rate;  /* -s: Alignment::filter rate (0.65) */
    uint32_t max_report;    /* -k: records per read (1); 0 for every alignment */
    int32_t n_threads;      /* host threads; 0 for all hardware threads */
    double gap_open, gap_ext, clip;  /* ScoreScheme gapO, gapE (5, 2) and clip penalty (4) */
} msg_tail_params;

void msg_tail_params_default(msg_tail_params* p);

/* One SAM record as msgseqtk-align writes it: exportBAM
 * (src/Alignment.cpp:429-444) plus output's flags and tags
 * (src/msgseqtk-align.cpp:538-556), or an unmapped record (flag 0x4, tid -1,
 * no CIGAR or tags; :583-585). SEQ and QUAL are the read's, reverse-
 * complemented and reversed when flag has 0x10. CIGAR words are the input
 * records' (cigar[cigar_off .. +n_cigar)); the MD:Z text is md[md_off ..
 * +md_len). XH:f and XP:f are float32 as the reference stores them. */
typedef struct msg_sam_rec {
    int64_t read;           /* read index in the batch */
    int32_t flag, tid;
    int64_t pos;            /* 0-based leftmost target position (alnStart) */
    int32_t mapq;
    int32_t as;             /* AS:i alignment score */
    float xh, xp;           /* XH:f log10 likelihood, XP:f posterior probability */
    int32_t nh, xn;         /* NH:i reported records of the read, XN:i alignments kept */
    int64_t cigar_off;
    int32_t n_cigar, md_len;
    int64_t md_off;
    int32_t isize;          /* TLEN: pairs only (AlignmentPE::exportFwdBAM/exportRevBAM) */
    int32_t pad;
} msg_sam_rec;

/* msgseqtk-align's per-read tail (src/msgseqtk-align.cpp:619-628): on each
 * read's records from msg_map_batch (aln, cigar, read_aln_off as returned),
 * Alignment::filter, evaluate, calcMapQ and sort (src/Alignment.cpp:446-555,
 * src/Alignment.h:629-633), then the reported records in output order. quals
 * holds phred values (not ASCII) at the reads' offsets (NULL: 33 on every
 * base, as PrimarySeq::fixQual gives reads without qualities); mtg
 * gives the forward chromosome sequences. Records go to out (out_cap), MD
 * texts to md (md_cap bytes); *n_out and *md_len receive the sizes needed,
 * and MSG_EINVAL is returned with nothing written when either exceeds its
 * capacity. Host memory only; threads as p->n_threads. */
int msg_tail_batch(const msg_mtg_view* mtg, const msg_read_batch* reads, const uint8_t* quals, const msg_aln* aln,
                   const uint32_t* cigar, const int64_t* read_aln_off, const msg_tail_params* p, msg_sam_rec* out,
                   int64_t out_cap, char* md, int64_t md_cap, int64_t* n_out, int64_t* md_len);

/* Pairing of msgseqtk-align's paired-end mode: AlignmentPE::ps as the
 * program leaves it after its options (-m/-d/-I/-X, src/msgseqtk-align.cpp:
 * 267-300, 400; an sd of 0 becomes mean * 0.1 and a mean of 0 makes every
 * insert size equally likely, PairingScheme::updateParam) and the pair
 * filters (--no-mixed, --no-discordant, --no-tail-over, --no-contain,
 * --no-overlap, --max-npair; 0 = no limit). The insert-size density is the
 * normal pdf exp(-z^2/2) / (sd sqrt(2 pi)). */
typedef struct msg_pair_params {
    double mean, sd, min_ins, max_ins;
    int32_t no_mixed, no_discordant, no_tail_over, no_contain, no_overlap;
    int32_t pad;
    int64_t max_npair;
} msg_pair_params;

/* Defaults: mean 200, sd 20, inserts [0, 400], no filters. */
void msg_pair_params_default(msg_pair_params* q);

/* msgseqtk-align's paired-end tail (src/msgseqtk-align.cpp:703-748) for
 * pairs whose mates are reads 2i and 2i+1 of the batch (n_reads even), on
 * their records from msg_map_batch: Alignment::filter and evaluate per mate,
 * AlignmentPE::getPairs/sort/filter/calcMapQ (src/Alignment.cpp:514-581) and
 * the pair records (flags 0x1|0x2|0x40/0x80, the pair's MAPQ and XP, TLEN),
 * or each mate's own records with flags 0x1|0x40/0x80 when no pair is left
 * (unless no_mixed), or two unmapped records (flags 77 and 141) when neither
 * mate keeps an alignment. Output as msg_tail_batch. */
int msg_tail_pe_batch(const msg_mtg_view* mtg, const msg_read_batch* reads, const uint8_t* quals,
                      const msg_aln* aln, const uint32_t* cigar, const int64_t* read_aln_off,
                      const msg_tail_params* p, const msg_pair_params* q, msg_sam_rec* out, int64_t out_cap,
                      char* md, int64_t md_cap, int64_t* n_out, int64_t* md_len);

/* ---- Reads in, SAM text out (host only) ---- */

/* Caller-owned buffers for msg_fastq_parse: nt16 codes and phred values of
 * the reads at off[i] .. off[i+1] (cap_bases each), and per read a text line
 * "name\tdescription\n" at text[name_off[i] .. name_off[i+1]) (cap_text
 * bytes); off and name_off hold cap_reads + 1 entries. */
typedef struct msg_fastq_batch {
    int64_t cap_reads, cap_bases, cap_text;
    uint8_t* seq;
    uint8_t* qual;
    int64_t* off;
    char* text;
    int64_t* name_off;
    int64_t n_reads, n_bases, n_text;  /* out */
} msg_fastq_batch;

/* FASTQ records from text[0 .. len) as msgseqtk-align's reader makes them
 * (while the next character is '@': SeqIO::nextFastqSeq, src/SeqIO.cpp:74-87):
 * the name is the first word after '@' (leading whitespace, newlines
 * included, skipped), the description the rest of that line after its
 * blanks, then the sequence line, the separator line and the quality line,
 * each up to '\n' ('\r' is kept as a character). Bases are encoded with
 * DNAalphabet's table (characters it does not list become 0), qualities as
 * max(uint8(c - 33), 2), and a quality string of another length is cut or
 * padded with 33 to the sequence's length (PrimarySeq::fixQual). Parsing
 * stops at the first record that does not fit the buffers, at the first
 * record whose four lines are not all in the text unless at_eof (then
 * missing lines are empty, as at the end of a stream), or at a line that
 * does not start with '@'. *consumed receives the bytes of the records
 * parsed, so a caller streams a file by passing the rest again. */
int msg_fastq_parse(const char* text, int64_t len, int at_eof, msg_fastq_batch* out, int64_t* consumed);

/* FASTQ text of the reads of a batch (those with keep[i] != 0; every read
 * when keep is NULL), as msgseqtk-clean writes the reads it keeps
 * (SeqIO::writeFastqSeq, src/SeqIO.cpp:107-116): "@name", " description"
 * when there is one, the bases decoded with DNAalphabet's symbols, "+", the
 * qualities + 33 (33 + 33 when quals is NULL). Names and descriptions come from msg_fastq_parse's
 * "name\tdescription\n" lines (text, name_off). Writes *text_len bytes into
 * out (cap bytes; MSG_EINVAL with *text_len set when they do not fit). */
int msg_fastq_format(const msg_read_batch* reads, const uint8_t* quals, const char* text, const int64_t* name_off,
                     const uint8_t* keep, char* out, int64_t cap, int64_t* text_len);

/* msgseqtk-clean's read-assignment lines (--assign; src/msgseqtk-clean.cpp:
 * 436-437, 473-474): "id\tdescription\trefLoglik\tbgLoglik\tLOD" per read,
 * the numbers as a C++ ostream prints a double by default, from
 * msg_fastq_parse's name lines and msg_clean_batch's outputs. The file's
 * header lines are the caller's. Writes *text_len bytes into out (cap bytes;
 * MSG_EINVAL with *text_len set when they do not fit). */
int msg_clean_format(const char* text, const int64_t* name_off, int64_t n, const double* ref_loglik,
                     const double* bg_loglik, const double* lod, char* out, int64_t cap, int64_t* text_len);

/* SAM text lines of msg_tail_batch / msg_tail_pe_batch records, laid out as
 * htslib's sam_format1 prints the BAM records msgseqtk-align writes: QNAME
 * (the read's name from its "name\tdescription" text line), FLAG, RNAME
 * (chrom_names[tid], '*' when unmapped), POS (pos + 1), MAPQ, CIGAR ('*'
 * when empty), RNEXT '*' and PNEXT 1 (the records' mate fields are left at
 * -1 and 0, src/SAMtools/BAM.h:61-75), TLEN, SEQ and QUAL (reverse-
 * complemented and reversed when flag has 0x10; phred + 33, and 33 + 33 for
 * every base when quals is NULL, as for reads without qualities), then AS:i, MD:Z,
 * XH:f, NH:i, XN:i, XP:f for mapped records, floats with %g (htslib's
 * exact float formatting is not pinned). Writes *text_len bytes into out
 * (cap bytes; MSG_EINVAL with *text_len set when they do not fit). */
int msg_sam_format(const msg_sam_rec* recs, int64_t n_recs, const char* md, const msg_read_batch* reads,
                   const uint8_t* quals, const uint32_t* cigar, const char* names, const int64_t* name_off,
                   const char* const* chrom_names, int64_t n_chrom, char* out, int64_t cap, int64_t* text_len);

/* BAM output (msgseqtk-align's `-o out.bam`, written through htslib in the
 * reference: src/msgseqtk-align.cpp:473-519, src/SAMtools/SAMfile.cpp), for
 * callers without htslib. A file is
 *   msg_bgzf_compress(header) + msg_bgzf_compress(records)... + the EOF member.
 *
 * msg_bam_header: the binary header of the SAM/BAM specification -- "BAM",
 * the header text as given (the caller's @HD/@SQ/@PG lines), and one
 * reference per chromosome (name, length) in tid order. */
int msg_bam_header(const char* text, int64_t text_len, const char* const* chrom_names, const int64_t* chrom_len,
                   int64_t n_chrom, uint8_t* out, int64_t cap, int64_t* len);

/* msg_bam_format: the binary records of msg_sam_format's lines, from the same
 * inputs -- the fields msgseqtk-align's BAM records carry (src/SAMtools/
 * BAM.cpp:20-56: bin from [pos, pos + reference length of the CIGAR), next
 * refID -1 and next pos 0, read name without padding, SEQ as nt16 codes two
 * per byte, QUAL as phred values) and the aux fields in the order the
 * reference sets them (AS, MD, XH, NH, XN, XP; integers in the smallest type
 * that holds them, as htslib's bam_aux_update_int stores them). Writes *len
 * bytes (uncompressed) into out (cap bytes; MSG_EINVAL with *len set when
 * they do not fit). */
int msg_bam_format(const msg_sam_rec* recs, int64_t n_recs, const char* md, const msg_read_batch* reads,
                   const uint8_t* quals, const uint32_t* cigar, const char* names, const int64_t* name_off,
                   int64_t n_chrom, uint8_t* out, int64_t cap, int64_t* len);

/* msg_bgzf_compress: data[0..n) as BGZF members of at most 0xff00 input bytes
 * each (raw deflate at `level` 0-9, CRC32 and size; the members are
 * compressed on up to n_threads host threads and written in order), followed
 * by the 28-byte end-of-file member when add_eof is set. Writes *len bytes
 * into out (cap bytes; MSG_EINVAL with *len set when they do not fit). */
int msg_bgzf_compress(const uint8_t* data, int64_t n, int level, int n_threads, int add_eof, uint8_t* out,
                      int64_t cap, int64_t* len);

/* ---- MEM search and read cleaning (msgseqtk-clean) ---- */

typedef struct msg_mem_params {
    int64_t min_len;        /* --min-seed, SMEM::MIN_LENGTH = 17 */
    double max_evalue;      /* --max-evalue, 0.01; +inf for no limit */
} msg_mem_params;

void msg_mem_params_default(msg_mem_params* p);

/* SMEM_LIST::findMEMS (src/SMEM.cpp:174-184, SMEM::findMEM :42-62) on each
 * read of a batch in HOST memory against the context's index, with
 * MEM_LIST::loglik (src/SMEM.cpp:307-312) of each read's list. loglik and
 * n_mem get n_reads entries (either may be NULL). rows (may be NULL): the MEMs
 * of all reads in read order, 6 int64 each (from, to, fwdStart, revStart,
 * size, logP bit pattern, the SMEM fields of src/SMEM.h:196-200); *n_rows
 * receives their count, and MSG_EINVAL is returned with rows untouched when it
 * exceeds row_cap. msg_last_stats afterwards: n_reads, n_smem (MEMs kept),
 * n_ext, n_launch, ms_smem (search) and ms_total. */
int msg_mem_batch(msg_ctx* ctx, const msg_read_batch* reads, const msg_mem_params* params, double* loglik,
                  int32_t* n_mem, int64_t* rows, int64_t row_cap, int64_t* n_rows);

/* msgseqtk-clean's per-read task (src/msgseqtk-clean.cpp:413-446 single-end,
 * :448-486 paired-end): findMEMS of each read against the reference genomes
 * (ref's index) and the background genomes (bg's index); refLoglik and
 * bgLoglik are the lists' loglik (for a pair, first mate's + second mate's,
 * src/SMEM.h:391-393); lod = -refLoglik + bgLoglik; keep = lod > min_lod.
 * fwd holds the reads (first mates), rev the second mates or NULL for
 * single-end data (same n_reads). Both contexts must live on the same device
 * with their indexes loaded; the call runs on ref's stream and reads bg's
 * index, so no other call may use bg meanwhile. Host outputs of n_reads
 * entries; any may be NULL. msg_last_stats(ref) as for msg_mem_batch. */
int msg_clean_batch(msg_ctx* ref, msg_ctx* bg, const msg_read_batch* fwd, const msg_read_batch* rev,
                    const msg_mem_params* params, double min_lod, double* ref_loglik, double* bg_loglik,
                    double* lod, uint8_t* keep);

/* Same with the reads already in device memory (seq and off of fwd and rev are
 * device pointers); results still land in the caller's host buffers. */
int msg_clean_batch_device(msg_ctx* ref, msg_ctx* bg, const msg_read_batch* dev_fwd,
                           const msg_read_batch* dev_rev, const msg_mem_params* params, double min_lod,
                           double* ref_loglik, double* bg_loglik, double* lod, uint8_t* keep);

/* ---- Single-operation entry points (parity checks of the index layer) ---- */

/* WaveletTreeRRR::rank (src/libsds/src/WaveletTreeRRR.cpp:101-125) through
 * FMDIndex: occurrences of nt16 symbol b[k] in BWT[0 .. i[k]] (or -1 when
 * i[k] >= n) for k < count. Host arrays. */
int msg_occ_query(msg_ctx* ctx, int64_t count, const uint8_t* b, const int64_t* i, int64_t* out);

/* FMDIndex::backExt (src/FMDIndex.cpp:577-610) when dir == 0, fwdExt
 * (src/FMDIndex.h:226-228) when dir == 1, on count bi-intervals in place;
 * ret[k] receives the returned size. Host arrays. */
int msg_bi_ext_query(msg_ctx* ctx, int64_t count, int dir, const uint8_t* b, int64_t* p, int64_t* q,
                     int64_t* s, int64_t* ret);

/* FMDIndex::accessSA (src/FMDIndex.cpp:520-527) for count rows. Host arrays. */
int msg_sa_query(msg_ctx* ctx, int64_t count, const int64_t* rows, int64_t* out);

#ifdef __cplusplus
}
#endif
#endif
