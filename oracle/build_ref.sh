#!/bin/sh
# Builds oracle/_ref/libksw_ref.so: the reference's own ksw_extend2, compiled from its
# source file where it lies (bwa/src/ksw.cu, lines 299-401 = eh_t + ksw_extend2) as host
# C++, the reference's own band-retry lines of mem_chain2aln (bwa/src/aux.cu:253-255,
# 258-301, 309), the whole of mem_chain2aln with the window fetch it calls
# (bwa/src/aux.cu:168-175, 178-315; bwa/src/bntseq.cu:5, 7-87), the banded global alignment
# with backtrack (bwa/src/ksw.cu:299-301, 548, 694-809) and the NM/MD block of the traceback
# stage (bwa/src/aux.cu:2830-2861), the striped local alignment ksw_align2 with ksw_qinit and
# ksw_i16 (bwa/src/ksw.cu:5, 18-292 less its trap line 276; bwa/src/ksw.h:7-29), the pair
# preparation of the traceback stage (bwa/src/aux.cu:506-513, 2698-2737; bwa/src/bntseq.cu:5,
# 39-60), the seed filter of long reads (bwa/src/aux.cu:117-162 with bwa/src/bntseq.cu:7-87),
# plus the ctypes batch driver ref_wrap.cpp.  The source lines are streamed from the
# reference tree into the compiler; no reference source is copied into this repository.
# Usage: sh oracle/build_ref.sh [reference_root]
#   (default: $G3X_REFERENCE, else a checkout named "reference" beside this repository)
set -eu
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${G3X_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}}
SRC="$REF/bwa/src/ksw.cu"
OUT="$HERE/_ref"
if [ ! -f "$SRC" ]; then
    echo "build_ref.sh: $SRC not found; oracle/_ref not built" >&2
    exit 2
fi
# Guard: the extracted range must be exactly the eh_t typedef and the ksw_extend2 body.
L299=$(sed -n '299p' "$SRC" | tr -d '\r')
L303=$(sed -n '303p' "$SRC" | tr -d '\r' | cut -c1-30)
L401=$(sed -n '401p' "$SRC" | tr -d '\r')
if [ "$L299" != "typedef struct {" ] || [ "$L303" != "__device__ int ksw_extend2(int" ] || [ "$L401" != "}" ]; then
    echo "build_ref.sh: unexpected content at ksw.cu:299/303/401; refusing to build" >&2
    exit 3
fi
mkdir -p "$OUT"
CXX=${CXX:-g++}
sed -n '299,401p' "$SRC" | tr -d '\r' | \
    $CXX -O3 -fPIC -x c++ -include "$HERE/ref_shim.h" -c - -o "$OUT/ksw_ref_fn.o"
# The band-retry driver: mem_chain2aln's left/right extension lines, unmodified, inside a
# host function whose locals ref_seed_head.inc declares.
AUX="$REF/bwa/src/aux.cu"
AUXH="$REF/bwa/src/aux.cuh"
A258=$(sed -n '258p' "$AUX" | tr -d '\r' | sed 's/^ *//')
A301=$(sed -n '301p' "$AUX" | tr -d '\r' | sed 's/^ *//')
A309=$(sed -n '309p' "$AUX" | tr -d '\r' | sed 's/^ *//')
if [ "$A258" != "if (s->qbeg) { // left extension" ] || \
   [ "$A301" != "} else a->qe = l_query, a->re = s->rbeg + s->len;" ] || \
   [ "$A309" != "a->w = aw[0] > aw[1]? aw[0] : aw[1];" ]; then
    echo "build_ref.sh: unexpected content at aux.cu:258/301/309; refusing to build" >&2
    exit 3
fi
{ grep -m1 '^#define MAX_BAND_TRY' "$AUXH"; cat "$HERE/ref_seed_head.inc"; \
  sed -n '253,255p;258,301p;309p' "$AUX"; echo '}'; } | tr -d '\r' | \
    $CXX -O3 -fPIC -x c++ -include "$HERE/ref_shim.h" -c - -o "$OUT/seed_ref_fn.o"
# The chain level: the reference's own mem_chain2aln with cal_max_gap (aux.cu:168-175,
# 178-315) and the window fetch it calls (bntseq.cu:5, 7-87), between ref_chain_head.inc and
# ref_chain_tail.inc.
BNS="$REF/bwa/src/bntseq.cu"
A168=$(sed -n '168p' "$AUX" | tr -d '\r')
A178=$(sed -n '178p' "$AUX" | tr -d '\r' | cut -c1-30)
A315=$(sed -n '315p' "$AUX" | tr -d '\r')
B5=$(sed -n '5p' "$BNS" | tr -d '\r' | cut -c1-16)
B7=$(sed -n '7p' "$BNS" | tr -d '\r')
B87=$(sed -n '87p' "$BNS" | tr -d '\r')
if [ "$A168" != "__device__ static inline int cal_max_gap(const mem_opt_t *opt, int qlen)" ] || \
   [ "$A178" != "__device__ void mem_chain2aln(" ] || [ "$A315" != "}" ] || \
   [ "$B5" != "#define _get_pac" ] || [ "$B7" != "__device__ int bns_pos2rid_gpu(const bntseq_t *bns, int64_t pos_f)" ] || \
   [ "$B87" != "}" ]; then
    echo "build_ref.sh: unexpected content at aux.cu:168/178/315 or bntseq.cu:5/7/87; refusing to build" >&2
    exit 3
fi
{ grep -m1 '^#define MAX_BAND_TRY' "$AUXH"; cat "$HERE/ref_chain_head.inc"; sed -n '5p;7,87p' "$BNS"; \
  sed -n '168,175p;178,315p' "$AUX"; cat "$HERE/ref_chain_tail.inc"; } | tr -d '\r' | \
    $CXX -O3 -fPIC -std=c++17 -x c++ -include "$HERE/ref_shim.h" -c - -o "$OUT/chain_ref_fn.o"
# Banded global alignment: eh_t, MINUS_INF, push_cigar and ksw_global2 (ksw.cu:299-301, 548,
# 694-704, 706-809) between ref_global_head.inc and ref_global_tail.inc.
K548=$(sed -n '548p' "$SRC" | tr -d '\r' | sed 's/^ *//')
K694=$(sed -n '694p' "$SRC" | tr -d '\r' | cut -c1-49)
K706=$(sed -n '706p' "$SRC" | tr -d '\r' | cut -c1-26)
K809=$(sed -n '809p' "$SRC" | tr -d '\r')
if [ "$K548" != "#define MINUS_INF -0x40000000" ] || [ "$K694" != "__device__ static inline uint32_t *push_cigar(int" ] || \
   [ "$K706" != "__device__ int ksw_global2" ] || [ "$K809" != "}" ]; then
    echo "build_ref.sh: unexpected content at ksw.cu:548/694/706/809; refusing to build" >&2
    exit 3
fi
{ cat "$HERE/ref_global_head.inc"; sed -n '299,301p;548p;694,704p;706,809p' "$SRC"; cat "$HERE/ref_global_tail.inc"; } | \
    tr -d '\r' | $CXX -O3 -fPIC -std=c++17 -x c++ -include "$HERE/ref_shim.h" -c - -o "$OUT/global_ref_fn.o"
# NM and MD of the traceback stage (aux.cu:2830-2861) inside the host function of
# ref_nmmd_head.inc / ref_nmmd_tail.inc.
A2830=$(sed -n '2830p' "$AUX" | tr -d '\r' | sed 's/^ *//')
A2862=$(sed -n '2862p' "$AUX" | tr -d '\r' | sed 's/^ *//')
if [ "$A2830" != "int NM;" ] || [ "$A2862" != "// write output" ]; then
    echo "build_ref.sh: unexpected content at aux.cu:2830/2862; refusing to build" >&2
    exit 3
fi
{ cat "$HERE/ref_nmmd_head.inc"; sed -n '2830,2861p' "$AUX"; cat "$HERE/ref_nmmd_tail.inc"; } | tr -d '\r' | \
    $CXX -O3 -fPIC -std=c++17 -x c++ -c - -o "$OUT/nmmd_ref_fn.o"
# Striped local alignment: ksw.h:7-29 (flags and types), ksw.cu:5 (g_defr), 18-275 and 277-292
# (ksw_qinit, the m128i helpers, ksw_i16, revseq, ksw_align2 without its trap line 276) between
# ref_sw_head.inc and ref_sw_tail.inc.
KSWH="$REF/bwa/src/ksw.h"
K5=$(sed -n '5p' "$SRC" | tr -d '\r' | cut -c1-32)
K18=$(sed -n '18p' "$SRC" | tr -d '\r' | cut -c1-35)
K155=$(sed -n '155p' "$SRC" | tr -d '\r' | cut -c1-33)
K271=$(sed -n '271p' "$SRC" | tr -d '\r' | cut -c1-29)
K276=$(sed -n '276p' "$SRC" | tr -d '\r')
K292=$(sed -n '292p' "$SRC" | tr -d '\r')
H7=$(sed -n '7p' "$KSWH" | tr -d '\r' | cut -c1-17)
H29=$(sed -n '29p' "$KSWH" | tr -d '\r')
if [ "$K5" != "__device__ const kswr_t g_defr =" ] || [ "$K18" != "static __device__ kswq_t* ksw_qinit" ] || \
   [ "$K155" != "static __device__ kswr_t ksw_i16(" ] || [ "$K271" != "__device__ kswr_t ksw_align2(" ] || \
   [ "$K276" != 'printf("this part of code for long reads is under development \n"); __trap();' ] || \
   [ "$K292" != "}" ] || [ "$H7" != "#define KSW_XBYTE" ] || [ "$H29" != "} kswr_t;" ]; then
    echo "build_ref.sh: unexpected content at ksw.cu:5/18/155/271/276/292 or ksw.h:7/29; refusing to build" >&2
    exit 3
fi
{ cat "$HERE/ref_sw_head.inc"; sed -n '7,29p' "$KSWH"; sed -n '5p;18,275p;277,292p' "$SRC"; cat "$HERE/ref_sw_tail.inc"; } | \
    tr -d '\r' | $CXX -O3 -fPIC -std=c++17 -x c++ -include "$HERE/ref_shim.h" -c - -o "$OUT/sw_ref_fn.o"
# Pair preparation of the traceback stage: bntseq.cu:5, 39-60 (_get_pac, bns_get_seq_gpu),
# aux.cu:506-513 (infer_bw) and the per-record lines of FINALIZEALN_preprocessing2_kernel
# (aux.cu:2698-2737) between ref_tbpair_head.inc, ref_tbpair_mid.inc and ref_tbpair_tail.inc.
T506=$(sed -n '506p' "$AUX" | tr -d '\r' | sed 's/^ *//;s/ *$//')
T513=$(sed -n '513p' "$AUX" | tr -d '\r' | sed 's/^ *//;s/ *$//')
T2698=$(sed -n '2698p' "$AUX" | tr -d '\r' | sed 's/^ *//;s/ *$//')
T2737=$(sed -n '2737p' "$AUX" | tr -d '\r' | sed 's/^ *//;s/ *$//')
B39=$(sed -n '39p' "$BNS" | tr -d '\r' | cut -c1-35)
B60=$(sed -n '60p' "$BNS" | tr -d '\r')
if [ "$T506" != "__device__ static inline int infer_bw(int l1, int l2, int score, int a, int q, int r)" ] || \
   [ "$T513" != "}" ] || [ "$T2698" != "int64_t rb = d_regs[seqID].a[alnID].rb;" ] || [ "$T2737" != "}" ] || \
   [ "$B39" != "__device__ uint8_t *bns_get_seq_gpu" ] || [ "$B60" != "}" ]; then
    echo "build_ref.sh: unexpected content at aux.cu:506/513/2698/2737 or bntseq.cu:39/60; refusing to build" >&2
    exit 3
fi
{ cat "$HERE/ref_tbpair_head.inc"; sed -n '5p;39,60p' "$BNS"; sed -n '506,513p' "$AUX"; cat "$HERE/ref_tbpair_mid.inc"; \
  sed -n '2698,2737p' "$AUX"; cat "$HERE/ref_tbpair_tail.inc"; } | tr -d '\r' | \
    $CXX -O3 -fPIC -std=c++17 -x c++ -include "$HERE/ref_shim.h" -c - -o "$OUT/tbpair_ref_fn.o"
# The seed filter of long reads: the MEM_SHORT_* / MEM_*_COEF constants (aux.cuh), ksw.h:7-31
# (flags, types, the ksw_align2 prototype), bntseq.cu:5, 7-87 (the window fetch) and
# aux.cu:117-162 (mem_seed_sw, mem_flt_chained_seeds) between ref_seedflt_head.inc and
# ref_seedflt_tail.inc; the call to ksw_align2 links to the unit above.
F117=$(sed -n '117p' "$AUX" | tr -d '\r' | cut -c1-27)
F143=$(sed -n '143p' "$AUX" | tr -d '\r')
F145=$(sed -n '145p' "$AUX" | tr -d '\r' | cut -c1-38)
F162=$(sed -n '162p' "$AUX" | tr -d '\r')
H31=$(sed -n '31p' "$KSWH" | tr -d '\r' | cut -c1-29)
if [ "$F117" != "__device__ int mem_seed_sw(" ] || [ "$F143" != "}" ] || \
   [ "$F145" != "__device__ void mem_flt_chained_seeds(" ] || [ "$F162" != "}" ] || \
   [ "$H31" != "__device__ kswr_t ksw_align2(" ]; then
    echo "build_ref.sh: unexpected content at aux.cu:117/143/145/162 or ksw.h:31; refusing to build" >&2
    exit 3
fi
{ cat "$HERE/ref_seedflt_head.inc"; \
  grep -m1 '^#define MEM_SHORT_EXT' "$AUXH"; grep -m1 '^#define MEM_SHORT_LEN' "$AUXH"; \
  grep -m1 '^#define MEM_HSP_COEF' "$AUXH"; grep -m1 '^#define MEM_MINSC_COEF' "$AUXH"; \
  grep -m1 '^#define MEM_SEEDSW_COEF' "$AUXH"; sed -n '7,31p' "$KSWH"; sed -n '5p;7,87p' "$BNS"; \
  sed -n '117,162p' "$AUX"; cat "$HERE/ref_seedflt_tail.inc"; } | tr -d '\r' | \
    $CXX -O3 -fPIC -std=c++17 -x c++ -include "$HERE/ref_shim.h" -c - -o "$OUT/seedflt_ref_fn.o"
$CXX -O3 -fPIC -shared -std=c++17 "$HERE/ref_wrap.cpp" "$OUT/ksw_ref_fn.o" "$OUT/seed_ref_fn.o" \
    "$OUT/chain_ref_fn.o" "$OUT/global_ref_fn.o" "$OUT/nmmd_ref_fn.o" "$OUT/sw_ref_fn.o" "$OUT/tbpair_ref_fn.o" \
    "$OUT/seedflt_ref_fn.o" -o "$OUT/libksw_ref.so" -lpthread
rm -f "$OUT/ksw_ref_fn.o" "$OUT/seed_ref_fn.o" "$OUT/chain_ref_fn.o" "$OUT/global_ref_fn.o" "$OUT/nmmd_ref_fn.o" \
    "$OUT/sw_ref_fn.o" "$OUT/tbpair_ref_fn.o" "$OUT/seedflt_ref_fn.o"
echo "built $OUT/libksw_ref.so"
