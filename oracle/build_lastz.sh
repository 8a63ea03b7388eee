#!/bin/sh
# Test infrastructure: builds signalAlign's vendored lastz (externalTools/lastz-distrib-1.03.54,
# installed by externalTools/Makefile:4-7 as cPecanLastz) from its own sources with gcc, for the
# anchor restatement in oracle/anchors.py that regenerates the banded known-answer fixtures.
# Nothing of the product uses it.  Outputs go to oracle/_ref/ only (git-ignored).
#
#   usage: oracle/build_lastz.sh /path/to/signalAlign     (or SIGNALALIGN_SRC set)
#
# The flags are the ones lastz's own src/Makefile uses for its integer-scoring build:
#   -O3 -Wall -Wextra -D_FILE_OFFSET_BITS=64 -D_LARGEFILE_SOURCE, the VERSION_* strings of
#   src/version.mak, and -Dscore_type='I'.
set -e
SRC_TREE=${1:-$SIGNALALIGN_SRC}
if [ -z "$SRC_TREE" ]; then
    echo "usage: $0 /path/to/signalAlign (or set SIGNALALIGN_SRC)" >&2
    exit 2
fi
LZ="$SRC_TREE/externalTools/lastz-distrib-1.03.54/src"
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
OBJ="$OUT/lastz_obj"
mkdir -p "$OBJ"
CFLAGS="-O3 -w -D_FILE_OFFSET_BITS=64 -D_LARGEFILE_SOURCE"
PARTS="lastz infer_scores seeds pos_table quantum seed_search diag_hash chain gapped_extend tweener masking
       segment edit_script identity_dist coverage_dist continuity_dist output gfa lav axt maf cigar sam
       genpaf text_align align_diffs utilities dna_utilities sequences capsule"
OBJS=""
for p in $PARTS; do
    gcc -c $CFLAGS -DVERSION_MAJOR='"1"' -DVERSION_MINOR='"03"' -DVERSION_SUBMINOR='"54"' \
        -DREVISION_DATE='"20140128"' -DSUBVERSION_REV='"1827:1830"' -Dscore_type="'I'" \
        -I"$LZ" "$LZ/$p.c" -o "$OBJ/$p.o"
    OBJS="$OBJS $OBJ/$p.o"
done
gcc $OBJS -lm -o "$OUT/cPecanLastz"
echo "built $OUT/cPecanLastz"
