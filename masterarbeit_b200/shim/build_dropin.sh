#!/usr/bin/env bash
# build_dropin.sh -- link the reference's own drivers against libsu2g through ref_shim.c.
#
# For each lattice size (T x X x Y x Z; the reference fixes it at compile time in
# LGT_Code/include/headers.h:22-25) this compiles, from the reference tree where it lies:
#   drivers   main/qcd.c, main_meas/meas.c, main_qtop/qtop.c        (unmodified)
#   modules   random, admin, io (config_IO with readConfig / writeConfig /
#             readConfigForThermalisation renamed ref_*), and for meas the fermion modules
#             (2pt with measure2ptFunctions renamed ref_*)
# and replaces the modules update, heatbath, metro, exp_fct, plaquette, smearing, wilson and
# topologicalcharge by ref_shim.c on top of libsu2g.so.  The header directory is copied into the
# build folder to patch the extents, because modules.h includes "headers.h" from its own
# directory.  Outputs go to masterarbeit_b200/shim/_build/<dims>/.
#
# usage: build_dropin.sh REF_ROOT [DIMS ...]
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
PKG="$(dirname "$HERE")"
REPO="$(dirname "$PKG")"
[ $# -ge 1 ] || { echo "usage: build_dropin.sh REF_ROOT [DIMS ...]" >&2; exit 2; }
REF="$1"
shift
DIMS=("$@")
[ ${#DIMS[@]} -eq 0 ] && DIMS=(8x8x8x8)
LGT="$REF/LGT_Code"
[ -f "$LGT/include/headers.h" ] || { echo "build_dropin.sh: no reference tree at $LGT" >&2; exit 1; }
LIB="$PKG/_lib/libsu2g.so"
[ -f "$LIB" ] || { echo "build_dropin.sh: build libsu2g.so first (python masterarbeit_b200/build.py)" >&2; exit 1; }

COMMON=(modules/random/random_su3.c modules/random/ranlxd.c
        modules/admin/init.c modules/admin/sun_vfunc.c modules/admin/endian.c
        modules/admin/error_checks.c modules/admin/utils.c
        modules/io/IO_utils.c modules/io/inp_IO.c)
FERMION=(modules/dirac/dirac_wil.c modules/dirac/spin_alg.c modules/dirac/sources.c modules/invert/solv_cg.c)
CFLAGS="-O3 -w -mcmodel=large"

for spec in "${DIMS[@]}"; do
    IFS=x read -r LT L1 L2 L3 <<<"$spec"
    OUT="$HERE/_build/$spec"
    rm -rf "$OUT"
    mkdir -p "$OUT/include" "$OUT/obj"
    cp "$LGT"/include/*.h "$OUT/include/"
    sed -i -E \
        -e "s/^#define LENGT [0-9]+UL/#define LENGT ${LT}UL/" \
        -e "s/^#define LENGS1 [0-9]+UL/#define LENGS1 ${L1}UL/" \
        -e "s/^#define LENGS2 [0-9]+UL/#define LENGS2 ${L2}UL/" \
        -e "s/^#define LENGS3 [0-9]+UL/#define LENGS3 ${L3}UL/" \
        "$OUT/include/headers.h"
    objs=()
    for m in "${COMMON[@]}" "${FERMION[@]}" modules/io/config_IO.c modules/obs/2pt.c; do
        o="$OUT/obj/$(basename "${m%.c}").o"
        gcc $CFLAGS -I"$OUT/include" -c "$LGT/$m" -o "$o" &
    done
    for d in main/qcd.c main_meas/meas.c main_qtop/qtop.c; do
        gcc $CFLAGS -I"$OUT/include" -c "$LGT/$d" -o "$OUT/obj/$(basename "${d%.c}").o" &
    done
    gcc $CFLAGS -I"$OUT/include" -I"$REPO/include" -c "$HERE/ref_shim.c" -o "$OUT/obj/ref_shim.o" &
    wait
    objcopy --redefine-sym readConfig=ref_readConfig --redefine-sym writeConfig=ref_writeConfig \
            --redefine-sym readConfigForThermalisation=ref_readConfigForThermalisation \
            "$OUT/obj/config_IO.o" "$OUT/obj/config_IO_ref.o"
    objcopy --redefine-sym measure2ptFunctions=ref_measure2ptFunctions "$OUT/obj/2pt.o" "$OUT/obj/2pt_ref.o"
    common_o=()
    for m in "${COMMON[@]}"; do common_o+=("$OUT/obj/$(basename "${m%.c}").o"); done
    fermion_o=()
    for m in "${FERMION[@]}"; do fermion_o+=("$OUT/obj/$(basename "${m%.c}").o"); done
    LINK=(-L"$PKG/_lib" -lsu2g -Wl,-rpath,'$ORIGIN/../../../_lib' -lm)
    gcc -mcmodel=large "$OUT/obj/qcd.o" "${common_o[@]}" "$OUT/obj/config_IO_ref.o" "$OUT/obj/ref_shim.o" \
        "${LINK[@]}" -o "$OUT/qcd"
    gcc -mcmodel=large "$OUT/obj/qtop.o" "${common_o[@]}" "$OUT/obj/config_IO_ref.o" "$OUT/obj/ref_shim.o" \
        "${LINK[@]}" -o "$OUT/qtop"
    gcc -mcmodel=large "$OUT/obj/meas.o" "${common_o[@]}" "$OUT/obj/config_IO_ref.o" "$OUT/obj/2pt_ref.o" \
        "${fermion_o[@]}" "$OUT/obj/ref_shim.o" "${LINK[@]}" -o "$OUT/meas"
    echo "built $OUT/{qcd,meas,qtop}"
done
