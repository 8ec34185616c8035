#!/bin/sh
# Compile the reference's own AdaTM files (where they lie in the reference
# checkout) with the SPLATT stand-in and the driver into one shared library.
#   build_ref.sh CC REF ARCH FLAGS OBJDIR OUTLIB "SRCS"
set -e
CC=$1; REF=$2; ARCH=$3; FLAGS=$4; OBJ=$5; OUT=$6; SRCS=$7
mkdir -p "$OBJ"
for f in $SRCS; do
  $CC $ARCH $FLAGS -c "$REF/src/$f" -o "$OBJ/${f%.c}.o"
done
$CC $ARCH $FLAGS -c ref_shim.c -o "$OBJ/ref_shim.o"
$CC $ARCH $FLAGS -c ref_driver.c -o "$OBJ/ref_driver.o"
$CC -O3 $ARCH -std=gnu99 -fopenmp -fPIC -c adatm_oracle.c -o "$OBJ/adatm_oracle.o"
$CC -shared -fopenmp -Wl,--wrap=mttkrp_csf_adaptive -o "$OUT" "$OBJ"/*.o -lm
rm -rf "$OBJ"
