#!/bin/sh
# Compiles the reference's C example plugins (hkbelagali/propaq,
# examples/plugins/c/{noise,truncation}/*.c) from the reference tree into
# oracle/_ref/, with the same flags the reference's notebooks use
# (examples/plugins/notebooks/02_rust_plugins.ipynb).  These plugins are test
# fixtures for the plugin ABI; nothing in the product links them.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# The reference tree: PROPAQ_REFERENCE, else a directory named `reference`
# beside the repository.
REF=${PROPAQ_REFERENCE:-$HERE/../../reference}
OUT="$HERE/_ref"
# Without the reference tree (the GPU box has only the prebuilt fixtures)
# there is nothing to build: --if-present makes that a quiet no-op.
if [ ! -d "$REF/examples/plugins/c" ]; then
  [ "$1" = "--if-present" ] && exit 0
  echo "reference tree not found at $REF" >&2
  exit 1
fi
mkdir -p "$OUT"
for src in "$REF"/examples/plugins/c/noise/*.c "$REF"/examples/plugins/c/truncation/*.c; do
  name=$(basename "$src" .c)
  gcc -shared -fPIC -O2 -o "$OUT/$name.so" "$src" -lm
done
ls "$OUT"
