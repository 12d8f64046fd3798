/* Stand-in for the reference's SAMtools/BAM.h (which needs htslib, absent
 * here), for the reference-oracle build only. It keeps the constructor and
 * setter signatures the reference Alignment code calls and records the SAM
 * core fields and aux tags as plain values. The CIGAR operation codes and
 * flag bits are the public SAM/BAM specification values. */
#ifndef MSG_SHIM_BAM_H
#define MSG_SHIM_BAM_H
#include <string>
#include <vector>
#include <cstdint>
#include <utility>

#define BAM_CMATCH 0
#define BAM_CINS 1
#define BAM_CDEL 2
#define BAM_CREF_SKIP 3
#define BAM_CSOFT_CLIP 4
#define BAM_CHARD_CLIP 5
#define BAM_CPAD 6
#define BAM_CEQUAL 7
#define BAM_CDIFF 8
#define BAM_CBACK 9
#define BAM_CIGAR_STR "MIDNSHP=XB"
#define BAM_CIGAR_SHIFT 4
#define BAM_CIGAR_MASK 0xf
#define bam_cigar_op(c) ((c) & BAM_CIGAR_MASK)
#define bam_cigar_oplen(c) ((c) >> BAM_CIGAR_SHIFT)
#define bam_cigar_opchr(c) (BAM_CIGAR_STR[bam_cigar_op(c)])
#define bam_cigar_gen(l, o) ((l) << BAM_CIGAR_SHIFT | (o))

#define BAM_FPAIRED 1
#define BAM_FPROPER_PAIR 2
#define BAM_FUNMAP 4
#define BAM_FMUNMAP 8
#define BAM_FREVERSE 16
#define BAM_FMREVERSE 32
#define BAM_FREAD1 64
#define BAM_FREAD2 128
#define BAM_FSECONDARY 256

namespace EGriceLab {
namespace SAMtools {
class BAM {
public:
    typedef std::basic_string<uint32_t> cigar_str;
    typedef std::basic_string<uint8_t> seq_str;
    typedef std::basic_string<uint8_t> qual_str;
    struct Aux { std::string tag; char type; double num; std::string str; };

    BAM() = default;
    BAM(const std::string& qname, uint16_t flag, int32_t tid, int32_t pos, uint8_t mapQ,
        const cigar_str& cigar, int32_t l_seq, const seq_str& seq, const qual_str& qual,
        int32_t mtid = -1, int32_t mpos = -1, int32_t isize = 0, size_t id = 0)
        : qname(qname), flag(flag), tid(tid), pos(pos), mapQ(mapQ), cigar(cigar), l_seq(l_seq),
          seq(seq), qual(qual), mtid(mtid), mpos(mpos), isize(isize) {}
    BAM(const std::string& qname, int32_t l_seq, const seq_str& seq, const qual_str& qual, uint16_t flag = 0)
        : BAM(qname, flag, -1, 0, 0, cigar_str(), l_seq, seq, qual) {}

    void setMapQ(uint8_t q) { mapQ = q; }
    uint16_t getFlag() const { return flag; }
    void setFlag(uint16_t f) { flag = f; }
    void setISize(int32_t s) { isize = s; }
    void setSecondaryFlag(bool f = true) { if (f) flag |= BAM_FSECONDARY; else flag &= ~BAM_FSECONDARY; }
    int setAux(const std::string& tag, int32_t v) { aux.push_back(Aux{tag, 'i', (double)v, ""}); return 0; }
    int setAux(const std::string& tag, uint32_t v) { aux.push_back(Aux{tag, 'i', (double)v, ""}); return 0; }
    int setAux(const std::string& tag, int64_t v) { aux.push_back(Aux{tag, 'i', (double)v, ""}); return 0; }
    int setAux(const std::string& tag, uint64_t v) { aux.push_back(Aux{tag, 'i', (double)v, ""}); return 0; }
    int setAux(const std::string& tag, float v) { aux.push_back(Aux{tag, 'f', (double)v, ""}); return 0; }
    int setAux(const std::string& tag, double v) { aux.push_back(Aux{tag, 'f', (double)(float)v, ""}); return 0; }
    int setAux(const std::string& tag, const std::string& v) { aux.push_back(Aux{tag, 'Z', 0, v}); return 0; }

    std::string qname;
    uint16_t flag = 0;
    int32_t tid = -1, pos = 0;
    uint8_t mapQ = 0;
    cigar_str cigar;
    int32_t l_seq = 0;
    seq_str seq;
    qual_str qual;
    int32_t mtid = -1, mpos = -1, isize = 0;
    std::vector<Aux> aux;
};
}  // namespace SAMtools
}  // namespace EGriceLab
#endif
