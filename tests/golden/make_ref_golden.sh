#!/bin/bash
# Runs the unmodified reference program (built by oracle/Makefile.ref) on a
# GPU for every case in ref_cases.py and keeps its text outputs.
#   bash tests/golden/make_ref_golden.sh <outdir> [spectra|snap]
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(cd "$HERE/../.." && pwd)"
if [ $# -lt 1 ]; then echo "usage: $0 <output directory> [spectra|snap]" >&2; exit 2; fi
OUT="$1"
SET="${2:-spectra}"
BIN="$ROOT/oracle/_ref/fdtd_ref"
test -x "$BIN"
python "$HERE/ref_cases.py" "$OUT" "$SET"
for d in "$OUT"/*/; do
  name=$(basename "$d")
  ( cd "$d" && mkdir -p videofiles && t0=$(date +%s%N) && timeout 600 "$BIN" > stdout.txt 2> stderr.txt; rc=$?; t1=$(date +%s%N); echo "rc=$rc" > rc.txt; echo "wall_ms=$(( (t1 - t0) / 1000000 ))" >> rc.txt ) || true
  # keep only what the fixtures need
  rm -f "$d"/Material_*.txt "$d"/SourceFile.txt "$d"/source.txt "$d"/Test.txt
  echo "$name: $(cat "$d/rc.txt" | tr '\n' ' ') $(tail -1 "$d/stderr.txt")"
done
