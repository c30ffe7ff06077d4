#!/usr/bin/env bash
# build_ref.sh -- compile the reference's own C sources into oracle/_ref/<T>x<X>x<Y>x<Z>/.
#
# ORACLE / TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline, never the product).
#
# The reference fixes the lattice size at compile time (LENGT, LENGS1-3 in
# LGT_Code/include/headers.h:22-25) and its modules.h includes "headers.h" from
# its own directory, so an -I override alone cannot change the size.  This
# recipe therefore copies the reference's header directory (headers only) into
# the build folder, patches the four extents there, and compiles every module
# .c file where it lies in the reference tree with -I pointing at that copy.
# Flags follow LGT_Code/main/Makefile:64-69,:85-98 (gcc -O3 -Wall -mcmodel=large).
# Shipped objects and binaries of the reference are never used.
#
# usage: oracle/build_ref.sh REF_ROOT [DIMS ...]     DIMS like 8x8x8x8 (T x X x Y x Z)
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
[ $# -ge 1 ] || { echo "usage: build_ref.sh REF_ROOT [DIMS ...]" >&2; exit 2; }
REF="$1"
shift
DIMS=("$@")
if [ ${#DIMS[@]} -eq 0 ]; then
    DIMS=(4x4x4x4 6x4x4x8 8x8x8x8 24x24x24x24 48x48x48x48)
fi
LGT="$REF/LGT_Code"
if [ ! -f "$LGT/include/headers.h" ]; then
    echo "build_ref.sh: reference tree not found at $LGT" >&2
    exit 1
fi

MODULES=(
  modules/random/random_su3.c
  modules/admin/init.c modules/admin/sun_vfunc.c modules/admin/endian.c
  modules/admin/error_checks.c modules/admin/utils.c
  modules/io/IO_utils.c modules/io/config_IO.c
  modules/update/update.c modules/update/metro.c modules/update/exp_fct.c modules/update/heatbath.c
  modules/obs/plaquette.c modules/obs/smearing.c modules/obs/wilson.c modules/obs/topologicalcharge.c
)

CFLAGS="-O3 -w -mcmodel=large"

# the reference's stand-alone autocorrelation tool (LGT_Code/Autocorrelation/t_int.c), unmodified
mkdir -p "$HERE/_ref"
if [ ! -x "$HERE/_ref/t_int" ] || [ "$LGT/Autocorrelation/t_int.c" -nt "$HERE/_ref/t_int" ]; then
    gcc -O2 -w "$LGT/Autocorrelation/t_int.c" -lm -o "$HERE/_ref/t_int"
fi

for spec in "${DIMS[@]}"; do
    IFS=x read -r LT L1 L2 L3 <<<"$spec"
    OUT="$HERE/_ref/$spec"
    if [ -x "$OUT/harness" ] && [ -x "$OUT/harness_inj" ] && [ "$OUT/harness" -nt "$HERE/ref_harness.c" ] \
       && [ "$OUT/harness_inj" -nt "$HERE/inject_ranlxd.c" ]; then
        continue
    fi
    rm -rf "$OUT"
    mkdir -p "$OUT/include" "$OUT/obj" "$OUT/obj_inj"
    cp "$LGT"/include/*.h "$OUT/include/"
    sed -i -E \
        -e "s/^#define LENGT [0-9]+UL/#define LENGT ${LT}UL/" \
        -e "s/^#define LENGS1 [0-9]+UL/#define LENGS1 ${L1}UL/" \
        -e "s/^#define LENGS2 [0-9]+UL/#define LENGS2 ${L2}UL/" \
        -e "s/^#define LENGS3 [0-9]+UL/#define LENGS3 ${L3}UL/" \
        "$OUT/include/headers.h"
    grep -q "^#define LENGT ${LT}UL" "$OUT/include/headers.h"
    objs=()
    for m in "${MODULES[@]}"; do
        o="$OUT/obj/$(basename "${m%.c}").o"
        gcc $CFLAGS -I"$OUT/include" -c "$LGT/$m" -o "$o" &
        objs+=("$o")
    done
    gcc $CFLAGS -I"$OUT/include" -c "$LGT/modules/random/ranlxd.c" -o "$OUT/obj/ranlxd.o" &
    gcc $CFLAGS -I"$OUT/include" -c "$HERE/ref_harness.c" -o "$OUT/obj/ref_harness.o" &
    gcc $CFLAGS -DSU2_INJECT -I"$OUT/include" -c "$HERE/ref_harness.c" -o "$OUT/obj_inj/ref_harness.o" &
    gcc $CFLAGS -I"$HERE" -c "$HERE/inject_ranlxd.c" -o "$OUT/obj_inj/inject_ranlxd.o" &
    wait
    gcc -mcmodel=large "$OUT/obj/ref_harness.o" "${objs[@]}" "$OUT/obj/ranlxd.o" -lm -o "$OUT/harness"
    gcc -mcmodel=large "$OUT/obj_inj/ref_harness.o" "${objs[@]}" "$OUT/obj_inj/inject_ranlxd.o" -lm \
        -o "$OUT/harness_inj"
    # the reference's own, unmodified drivers (main/qcd.c, main_meas/meas.c, main_qtop/qtop.c)
    extra=(modules/io/inp_IO.c modules/obs/2pt.c modules/dirac/dirac_wil.c modules/dirac/spin_alg.c
           modules/dirac/sources.c modules/invert/solv_cg.c)
    xobjs=()
    for m in "${extra[@]}"; do
        o="$OUT/obj/$(basename "${m%.c}").o"
        gcc $CFLAGS -I"$OUT/include" -c "$LGT/$m" -o "$o" &
        xobjs+=("$o")
    done
    for d in main/qcd.c main_meas/meas.c main_qtop/qtop.c; do
        gcc $CFLAGS -I"$OUT/include" -c "$LGT/$d" -o "$OUT/obj/$(basename "${d%.c}").o" &
    done
    wait
    for d in qcd meas qtop; do
        gcc -mcmodel=large "$OUT/obj/$d.o" "${objs[@]}" "$OUT/obj/ranlxd.o" "${xobjs[@]}" -lm -o "$OUT/$d"
    done
    echo "built $OUT"
done
