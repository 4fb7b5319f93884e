#!/bin/bash
# Runs the reference's GPU stage programs (compiled by oracle/ref_gpu.mk into oracle/_ref/gpu/)
# and this library's stage drivers of the same names (cupythia_b200/bin/), each with its default
# arguments, one after the other on the current GPU, inside the work directory given (the
# programs write events.lhe into their working directory).  Test infrastructure: the
# "reference on the same box" measurement; per-kernel device times come from running this
# script under `ncu --metrics gpu__time_duration.sum`.
#
# Output: <work dir>/{ref,ours}_<program>.log and one summary line per run on stdout.
# Exit status: 0 when every program ran to its VALIDATION line (PASS or FAIL, exit 0 or 2),
# 1 when any program reported a CUDA error or died.
#
# Usage: bash oracle/ref_gpu_run.sh <work dir>
set -u
ROOT=$(cd "$(dirname "$0")/.." && pwd)
W=${1:?usage: ref_gpu_run.sh <work dir>}
mkdir -p "$W"
W=$(cd "$W" && pwd)
PROGS="fused_gg2gg fp32_gg2gg vegas cub_compaction unweight_lhe pdf_xsec generate"
bad=0
for side in ref ours; do
  if [ "$side" = ref ]; then BIN="$ROOT/oracle/_ref/gpu"; else BIN="$ROOT/cupythia_b200/bin"; fi
  for p in $PROGS; do
    [ -x "$BIN/$p" ] || { echo "$side $p: not built"; continue; }
    [ "$side" = ours ] && [ ! -x "$ROOT/oracle/_ref/gpu/$p" ] && continue
    t0=$(date +%s.%N)
    (cd "$W" && "$BIN/$p") > "$W/${side}_$p.log" 2>&1
    rc=$?
    t1=$(date +%s.%N)
    v=$(grep -o "VALIDATION: [A-Z]*" "$W/${side}_$p.log" | head -1)
    printf '%s %s: exit %d, %s, %s s wall\n' "$side" "$p" "$rc" "${v:-no VALIDATION line}" \
      "$(awk -v a="$t0" -v b="$t1" 'BEGIN { printf "%.2f", b - a }')"
    if [ $rc -ne 0 ] && [ $rc -ne 2 ]; then bad=1; fi
    if grep -q "CUDA error" "$W/${side}_$p.log"; then bad=1; fi
  done
done
exit $bad
