#!/usr/bin/env bash
# Build the reference C library from its own sources (read in place under the
# reference checkout, never copied) into oracle/_ref/libnrLDPC_ref.so.
#
# The decoders keep their beliefs in file-static arrays; four small shim
# translation units #include the decoder sources and export accessors for
# those arrays so tests can compare final APP LLRs.  Flags follow the
# reference Makefile (c_lib/Makefile: -O3 -Wall -Wextra -fPIC).
#
# usage: oracle/build_ref.sh [reference-root]
#        (default: $NRLDPC_REFERENCE_ROOT, else /root/reference)
set -euo pipefail
REF="${1:-${NRLDPC_REFERENCE_ROOT:-/root/reference}}"
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
         BG2_trained_ldpc_weights.c c_ldpc_5g_decoder.c c_ldpc_5g_encoder.c \
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

# The channel model, wrapped so its static QAM mapper, max-log demapper and
# quantiser can be called on given symbols (the device front-end and the numpy
# restatement are pinned to them).  ref_demap_symbols computes the noise
# variance as tx_rx_process does and applies demodulate_symbol, then
# quantize_llr_to_int16, to each given noisy symbol.
cat > "$TMP/shim_channel.c" <<SHIM
#include "$SRC/tx_rx_process.c"
void ref_modulate_symbols(const uint8_t *bits, size_t n, uint16_t Qm, float *sym) {
  for (size_t i = 0; i < n; i++) {
    complex_float_t s = modulate_symbol(bits + i * Qm, Qm);
    sym[2 * i] = s.re;
    sym[2 * i + 1] = s.im;
  }
}
void ref_demap_symbols(const float *sym, size_t n, uint16_t Qm, float noise_power_db, int16_t *llr_out,
                       float *llr_float) {
  float noise_var = powf(10.0f, noise_power_db / 10.0f);
  for (size_t i = 0; i < n; i++) {
    complex_float_t s = {sym[2 * i], sym[2 * i + 1]};
    float l[8];
    demodulate_symbol(s, Qm, noise_var, l);
    for (uint16_t j = 0; j < Qm; j++) {
      llr_out[i * Qm + j] = quantize_llr_to_int16(l[j]);
      if (llr_float) llr_float[i * Qm + j] = l[j];
    }
  }
}
SHIM
$CC $CFLAGS -c "$TMP/shim_channel.c" -o "$TMP/shim_channel.o"

$CC -shared -o "$OUT/libnrLDPC_ref.so" "$TMP"/*.o -lm
echo "$OUT/libnrLDPC_ref.so"
