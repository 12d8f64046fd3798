/*
 * CPU restatement of MSGseqTK v1.2.3's read-mapping hot path (TEST
 * INFRASTRUCTURE: the checker for the CUDA path; nothing in the product links
 * it). Each function cites the reference file:line it follows. It works on the
 * decoded FMD-index view (BWT codes, base counts, the reference's own SA sample
 * set) and the chromosome table, i.e. the same inputs the CUDA library gets.
 *
 * Parity of this restatement is pinned against the reference compiled from its
 * own sources (oracle/_ref/libmsgref.so, built by oracle/ref/Makefile) and
 * against the committed fixtures under tests/golden/.
 */
#ifndef MSG_ORACLE_H
#define MSG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_index orc_index;

/* Index view: n BWT symbols (nt16 codes 0/1/2/4/8/15), B[16] base counts,
 * the reference's SA samples (rows sorted ascending, values), chromosome table
 * (BD start/end, forward length) and forward chromosome sequences (nt16,
 * concatenated at chr_off[t]..chr_off[t+1]). */
orc_index* orc_index_create(int64_t n, const uint8_t* bwt, const int64_t* B16,
                            int64_t n_samples, const int64_t* sample_rows, const int64_t* sample_vals,
                            int64_t n_chrom, const int64_t* bd_start, const int64_t* bd_end,
                            const int64_t* chr_len, const uint8_t* chr_seq, const int64_t* chr_off);
void orc_index_free(orc_index* ix);

int64_t orc_rank(const orc_index* ix, int b, int64_t i);
int64_t orc_back_ext(const orc_index* ix, int64_t* p, int64_t* q, int64_t* s, int b);
int64_t orc_fwd_ext(const orc_index* ix, int64_t* p, int64_t* q, int64_t* s, int b);
int64_t orc_access_sa(const orc_index* ix, int64_t i);
double orc_loglik(const orc_index* ix, int b);

/* SMEM_LIST::findAllSMEMS in emission order; rows of 6 int64:
 * from, to, fwdStart, revStart, size, logP (bit pattern). Returns count. */
int64_t orc_find_smems(const orc_index* ix, const uint8_t* read, int64_t L, int64_t min_len,
                       double max_evalue, int64_t* out, int64_t cap);

/* SMEM_LIST::findMEMS (msgseqtk-clean's search); rows of 6 int64 as for
 * SMEMs; *loglik receives SMEM_LIST::loglik of the list. Returns count. */
int64_t orc_find_mems(const orc_index* ix, const uint8_t* read, int64_t L, int64_t min_len,
                      double max_evalue, int64_t* out, int64_t cap, double* loglik);

/* SMEM_LIST::findSeeds; rows of 6 int64: from, to, start, end, tid, strand. */
int64_t orc_find_seeds(const orc_index* ix, const uint8_t* read, int64_t L, int64_t min_len,
                       double max_evalue, int64_t max_nseed, int64_t* out, int64_t cap);

/* SeedChain::getChains over seed rows (6 int64 each); chain k holds seed
 * indices out_idx[out_off[k] .. out_off[k+1]). Returns chain count. */
int64_t orc_get_chains(const int64_t* seeds, int64_t n, int64_t max_mismatch, int64_t max_indel,
                       int64_t* out_off, int64_t* out_idx, int64_t cap_chain, int64_t cap_idx);

/* One alignment per chain (Alignment::buildAlignments, before filter). */
typedef struct orc_aln {
    int64_t tid, strand, t_start, t_end, aln_from, aln_to, aln_start, aln_end;
    double aln_score;
    int64_t n_cigar, cigar_off, md_off, md_len;
    int64_t flags; /* bit0: last row had no finite cell; bit1: traceback left the matrix */
} orc_aln;

/* Align the given chain (seed rows of 6, in chain order) of a read
 * (mode 0 = GLOBAL/NW, 1 = LOCAL/SW) with integer score scheme
 * (match, mismatch, gap_open, gap_ext). */
int orc_align_chain(const orc_index* ix, const uint8_t* read, int64_t L, const int64_t* chain_seeds,
                    int64_t n_seeds, int mode, const int32_t* score4, orc_aln* out,
                    uint32_t* cigar_buf, int64_t cigar_cap, int64_t* cigar_used,
                    char* md_buf, int64_t md_cap, int64_t* md_used);

/* Whole per-read SE path through chain DP: seeds -> chains -> alignments
 * (msgseqtk-align.cpp:612-625). Returns the number of alignments. */
int64_t orc_align_read(const orc_index* ix, const uint8_t* read, int64_t L, int64_t min_len,
                       double max_evalue, int64_t max_nseed, int mode, const int32_t* score4,
                       orc_aln* out, int64_t cap, uint32_t* cigar_buf, int64_t cigar_cap,
                       int64_t* cigar_used, char* md_buf, int64_t md_cap, int64_t* md_used);

/* Batch of reads over n_threads std::threads (timing of the restated path). */
int64_t orc_map_batch(const orc_index* ix, int64_t n_reads, const uint8_t* reads, const int64_t* offs,
                      int64_t min_len, double max_evalue, int64_t max_nseed, int n_threads,
                      int64_t* n_aln_out, int64_t* n_cells_out);

#ifdef __cplusplus
}
#endif
#endif
