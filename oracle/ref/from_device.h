/*
 * from_device.h -- the reference's Alignment objects (src/Alignment.h) from
 * the records of the B200 library (msg_aln, include/msg_b200.h): the adapter a
 * maintainer adds to msgseqtk-align so that the reference's own per-read tail
 * (Alignment::filter, evaluate, calcMapQ, sort, exportBAM and the program's
 * output) runs unchanged on the records msg_map_batch returns.
 *
 * In the reference it belongs in src/Alignment.h as a static member,
 * `Alignment::fromDevice`, because it sets private fields. Compiled here
 * against the unmodified headers, the translation unit that includes it makes
 * those fields visible itself (private and protected defined as public before
 * the reference's headers); the function body is the same either way.
 * oracle/ref/ref_harness.cpp uses it for every comparison of GPU records with
 * the reference's SAM fields.
 */
#ifndef MSG_FROM_DEVICE_H
#define MSG_FROM_DEVICE_H
#include <cstdint>
#include <limits>

#include "Alignment.h"
#include "MetaGenome.h"
#include "msg_b200.h"

namespace msg_adapter {

/* The fields Alignment's chain constructor and buildAlignments set
 * (src/Alignment.h:84-94, src/Alignment.cpp:420-427) from one record: tid,
 * query strand, qFrom = 0, qTo = read length, the DP window tStart/tEnd,
 * alnFrom/To/Start/End, alnScore as a double (-inf for a record whose last row
 * held no finite score), and alnPath rebuilt from the CIGAR's M/I/D runs
 * (soft clips are alnFrom and alnTo). The DP matrices stay empty: nothing in
 * the tail reads them. */
inline EGriceLab::MSGseqTK::Alignment fromDevice(const EGriceLab::MSGseqTK::PrimarySeq* read,
                                                 const EGriceLab::MSGseqTK::PrimarySeq* rcRead,
                                                 const EGriceLab::MSGseqTK::MetaGenome& mtg, const msg_aln& rec,
                                                 const uint32_t* cigar,
                                                 EGriceLab::MSGseqTK::Alignment::MODE mode) {
    using namespace EGriceLab::MSGseqTK;
    Alignment a(read);
    a.rcRead = rcRead;
    a.tid = rec.tid;
    a.target = &mtg.getSeq(rec.tid);
    a.qStrand = (GLoc::STRAND)rec.strand;
    a.qFrom = 0;
    a.qTo = (int64_t)read->length();
    a.tStart = rec.t_start;
    a.tEnd = rec.t_end;
    a.alnMode = mode;
    a.alnFrom = rec.aln_from;
    a.alnTo = rec.aln_to;
    a.alnStart = rec.aln_start;
    a.alnEnd = rec.aln_end;
    a.alnScore = rec.aln_score == INT32_MIN ? -std::numeric_limits<double>::infinity() : (double)rec.aln_score;
    for (int32_t w = 0; w < rec.n_cigar; ++w) {
        const uint32_t c = cigar[rec.cigar_off + w];
        if ((c & 0xf) == BAM_CSOFT_CLIP) continue;
        a.alnPath.append(c >> 4, c & 0xf);
    }
    return a;
}

}  // namespace msg_adapter
#endif
