#!/usr/bin/env bash
# Build the reference C library from its own sources (read in place under the
# reference checkout, never copied) into oracle/_ref/libnrLDPC_ref.so.
#
# The decoders keep their beliefs in file-static arrays; four small shim
# translation units #include the decoder sources and export accessors for
# those arrays so tests can compare final APP LLRs.  Flags follow the
# reference Makefile (c_lib/Makefile: -O3 -Wall -Wextra -fPIC).
#
# usage: oracle/build_ref.sh [reference-root]   (default /root/reference)
set -euo pipefail
REF="${1:-/root/reference}"
SRC="$REF/c_lib"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$SRC/nr_ldpc.h" ]; then
  echo "reference sources not found under $SRC" >&2
  exit 2
fi
mkdir -p "$OUT"
CC="${CC:-gcc}"
CFLAGS="-O3 -fPIC -w -I$SRC"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT

# Sources compiled as they are.
for f in nr_crc.c ldpc_tables.c ldpc_internal.c ldpc_rate_recovery.c BG1_trained_ldpc_weights.c \
         BG2_trained_ldpc_weights.c c_ldpc_5g_decoder.c c_ldpc_5g_encoder.c tx_rx_process.c \
         ldpc_rate_match.c ldpc_encoder.c; do
  $CC $CFLAGS -c "$SRC/$f" -o "$TMP/${f%.c}.o"
done

# Decoder sources, each wrapped so its static belief array can be read.
shim() {  # name source accessor array type
  cat > "$TMP/shim_$1.c" <<EOF
#include "$SRC/$2"
$5 *$3(void) { return $4; }
EOF
  $CC $CFLAGS -c "$TMP/shim_$1.c" -o "$TMP/shim_$1.o"
}
shim fixed fixedpoint_ldpc_decoder.c ref_fixed_lq LQ int16_t
shim degree degree_fixedpoint_ldpc_decoder.c ref_degree_lq degree_LQ int16_t
shim neural neural_fixedpoint_ldpc_decoder.c ref_neural_lq neural_LQ int16_t
shim float floatpoint_ldpc_decoder.c ref_float_lq LQ float

$CC -shared -o "$OUT/libnrLDPC_ref.so" "$TMP"/*.o -lm
echo "$OUT/libnrLDPC_ref.so"
