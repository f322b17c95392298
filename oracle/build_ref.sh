#!/bin/sh
# Builds the reference CPU Tracker from its own sources into oracle/_ref/ (git-ignored).
#
# TEST INFRASTRUCTURE ONLY. The reference sources are read where they lie (ITSU_REFERENCE,
# default: a checkout named "reference" beside this repository); a patched working copy is written to oracle/_ref/src/ and compiled
# with the reference's own flags (-std=c++11 -O3, no -march, so no FMA contraction on x86-64).
# Patches (each a memory-safety or determinism fix; each sed is checked to apply exactly once):
#   P1 Tracker.cxx:88      candidate loop also stops at the end of the next layer
#   P2 Tracker.cxx:131     cells lookup table of layer L grown to the tracklets of layer L
#   P3 PVC.cxx:52          std::stable_sort instead of std::sort
#   P5 Tracker.cxx:84      a phi row's upper bin index clamped to 400
#   P4 (ref_cr only)       atan2f resolved to the correctly rounded itsu_atan2f
# Binaries: ref_cr (P1-P5), ref_stock (P1-P3, P5: the C library's atan2f) and
# ref_unstable (P1, P2, P4, P5: the reference's unstable std::sort); merge_pileup, the
# reference's pile-up merger (benchmarks/scripts/root/generatePileUpData.cxx), unpatched; and,
# when the library is built, ref_b200 (P1-P5 plus B1, B2: the B200 backend behind the
# reference's seam).
set -eu
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${ITSU_REFERENCE:-$HERE/../../reference}
OUT="$HERE/_ref"
CXX=${CXX:-g++}

if [ ! -f "$REF/src/CA/Tracker.cxx" ]; then
  echo "build_ref.sh: reference sources not found under $REF" >&2
  exit 2
fi

rm -rf "$OUT/src" "$OUT/src_unstable"
mkdir -p "$OUT/src"
cp "$REF"/src/CA/*.cxx "$OUT/src/"

apply() { # file, sed expression, expected pattern after the edit
  sed -i "$2" "$1"
  n=$(grep -c -F "$3" "$1" || true)
  if [ "$n" != "1" ]; then
    echo "build_ref.sh: patch did not apply once to $1 ($3): $n" >&2
    exit 3
  fi
}

T="$OUT/src/Tracker.cxx"
apply "$T" 's/iNextLayerCluster <= maxRowClusterIndex;/iNextLayerCluster <= maxRowClusterIndex \&\& iNextLayerCluster < static_cast<int>(primaryVertexContext.getClusters()[iLayer + 1].size()); \/\* P1 \*\//' '/* P1 */'
apply "$T" 's/const int maxBinIndex { firstBinIndex + selectedBinsRect.z - selectedBinsRect.x + 1 };/const int maxBinIndex { std::min(firstBinIndex + selectedBinsRect.z - selectedBinsRect.x + 1, Constants::IndexTable::ZBins * Constants::IndexTable::PhiBins) }; \/\* P5 \*\//' '/* P5 */'
apply "$T" 's/^\(    const int currentLayerTrackletsNum { static_cast<int>(primaryVertexContext.getTracklets()\[iLayer\].size()) };\)$/\1 if (iLayer > 0 \&\& static_cast<int>(primaryVertexContext.getCellsLookupTable()[iLayer - 1].size()) < currentLayerTrackletsNum) primaryVertexContext.getCellsLookupTable()[iLayer - 1].resize(currentLayerTrackletsNum, Constants::ITS::UnusedIndex); \/\* P2 \*\//' '/* P2 */'

cp -r "$OUT/src" "$OUT/src_unstable"
apply "$OUT/src/PrimaryVertexContext.cxx" 's/std::sort(mClusters\[iLayer\].begin(), mClusters\[iLayer\].end(), \[\](Cluster& cluster1, Cluster& cluster2)/std::stable_sort(mClusters[iLayer].begin(), mClusters[iLayer].end(), [](const Cluster\& cluster1, const Cluster\& cluster2) \/\* P3 \*\//' '/* P3 */'

FLAGS="-std=c++11 -O3 -ffp-contract=off -I$REF/include"
HARNESS="$HERE/ref_harness.cpp"
gcc -std=c99 -O2 -ffp-contract=off -c "$HERE/ref_atan2f.c" -o "$OUT/ref_atan2f.o"
$CXX $FLAGS -I"$HERE/../include" "$HARNESS" "$OUT"/src/*.cxx "$OUT/ref_atan2f.o" -o "$OUT/ref_cr" -DITSU_REF_CR=1
$CXX $FLAGS -I"$HERE/../include" "$HARNESS" "$OUT"/src/*.cxx -o "$OUT/ref_stock"
$CXX $FLAGS -I"$HERE/../include" "$HARNESS" "$OUT"/src_unstable/*.cxx "$OUT/ref_atan2f.o" -o "$OUT/ref_unstable" -DITSU_REF_CR=1
# ref_b200: the reference tracker with the B200 backend behind its own seam
# (tracking-itsu_b200/host/reference_backend/TrackerB200.cxx, linked against libitsu_b200.so), built
# from the P1-P3/P5 copy with the two edits that select the backend, each guarded by
# TRACKINGITSU_B200:
#   B1 Tracker.cxx:43    the CPU bodies of computeLayerTracklets / computeLayerCells are left out
#   B2 PVC.cxx:141       the CPU branch of initialize ends with the device clustering (b200Initialize)
LIB="$HERE/../tracking-itsu_b200/lib"
if [ -f "$LIB/libitsu_b200.so" ]; then
  rm -rf "$OUT/src_b200"
  cp -r "$OUT/src" "$OUT/src_b200"
  apply "$OUT/src_b200/Tracker.cxx" '0,/^#if !TRACKINGITSU_GPU_MODE$/s//#if !TRACKINGITSU_GPU_MODE \&\& !defined(TRACKINGITSU_B200) \/\* B1 \*\//' '/* B1 */'
  apply "$OUT/src_b200/PrimaryVertexContext.cxx" 's/^#endif$/#if defined(TRACKINGITSU_B200)\n  void b200Initialize(PrimaryVertexContext\&, const Event\&, int); \/\* B2 \*\/\n  b200Initialize(*this, event, primaryVertexIndex);\n#endif\n#endif/' '/* B2 */'
  $CXX $FLAGS -Wall -DTRACKINGITSU_B200 -I"$HERE/../include" "$HARNESS" "$OUT"/src_b200/*.cxx \
    "$HERE/../tracking-itsu_b200/host/reference_backend/TrackerB200.cxx" "$OUT/ref_atan2f.o" -DITSU_REF_CR=1 \
    -L"$LIB" -litsu_b200 -Wl,-rpath,'$ORIGIN/../../tracking-itsu_b200/lib' -o "$OUT/ref_b200"
  B200_BUILT=" $OUT/ref_b200"
else
  B200_BUILT=""
fi
# the reference's pile-up merger (a standalone program): merged_data.txt / merged_labels.txt
$CXX -std=c++11 -O2 "$REF/benchmarks/scripts/root/generatePileUpData.cxx" -o "$OUT/merge_pileup"
echo "built $OUT/ref_cr $OUT/ref_stock $OUT/ref_unstable $OUT/merge_pileup$B200_BUILT"
