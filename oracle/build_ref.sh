#!/usr/bin/env bash
# Build the reference's own CPU integrator (cuda/c_baseline) from the sources
# where they lie under the reference checkout, once per network plug-in and
# precision, into oracle/_ref/.  Nothing is copied into this repository: the
# reference .c files are compiled in place, and the only generated file is a
# per-network ode_gold.h (the reference header with NUM_CONST set to the
# network's constant count, which the reference leaves at 2 in
# cuda/include/ode_gold.h:12).
#
#   f64: -Dfloat=double  (the FP64 oracle build; bit-exact target)
#   f32: as shipped      (float state)
#
# Output: oracle/_ref/{sie,rk2}_gold_<net>_<prec>.so exporting
# goldIntegrateSystem (cuda/c_baseline/sie/sie_gold.c:81, rk2/rk2_gold.c:48).
set -euo pipefail
REF=${WIND_REFERENCE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
CB=$REF/cuda/c_baseline
if [ ! -f "$CB/common/common_gold.c" ]; then
    echo "build_ref.sh: reference sources not found under $REF" >&2
    exit 3
fi
mkdir -p "$OUT"
CC=${CC:-gcc}
# -ffp-contract=off: no FMA contraction, so products round before the add,
# as on the reference's x86-64 target and in the CUDA kernels.
BASE="-O2 -fPIC -shared -ffp-contract=off -DADAPTIVE_TIMESTEP -w"

gen_header () {   # $1 = dir, $2 = NUM_CONST
    mkdir -p "$1"
    sed -e "s/^#define NUM_CONST .*/#define NUM_CONST $2/" "$REF/cuda/include/ode_gold.h" > "$1/ode_gold.h"
}

build_net () {    # $1 = name, $2 = NUM_CONST, $3 = plugin source, $4 = extra defines
    local name=$1 nconst=$2 plugin=$3 extra=${4:-}
    local inc=$OUT/inc_$name
    gen_header "$inc" "$nconst"
    for prec in f64 f32; do
        local pflag=""
        [ "$prec" = f64 ] && pflag="-Dfloat=double"
        $CC $BASE $pflag -DSIE $extra -I"$inc" -I"$CB/include" -I"$REF/cuda/include" \
            "$CB/common/common_gold.c" "$CB/sie/sie_gold.c" \
            "$CB/linear_algebra/gje_gold.c" "$CB/linear_algebra/matrix_ops.c" \
            "$plugin" -o "$OUT/sie_gold_${name}_${prec}.so" -lm
        $CC $BASE $pflag -DRK2 $extra -I"$inc" -I"$CB/include" -I"$REF/cuda/include" \
            "$CB/common/common_gold.c" "$CB/rk2/rk2_gold.c" \
            "$plugin" -o "$OUT/rk2_gold_${name}_${prec}.so" -lm
    done
}

# Reference plug-in instances
build_net katz96 10 "$REF/cuda/ode_system/ode_gold.c"
build_net nr_test 4 "$HERE/plugins/nr_test_gold.c"
build_net stifftrig 2 "$HERE/plugins/stifftrig_gold.c"
# Katz96 tiled by the Precompiler's Ntile (one system of Ntile copies)
for nt in 3 8; do
    build_net "katz96_t$nt" 10 "$HERE/plugins/katz96_tiled_gold.c" "-DNTILE=$nt"
done
# Mass-action networks: ma_n<N>_r<R>[_lin]
for spec in "5 50 0" "16 160 0" "32 320 0" "64 640 0" "157 1570 0" "32 64 1" \
            "3 6 1" "8 20 0" "12 30 1"; do
    set -- $spec
    N=$1; R=$2; LIN=$3
    nc=$((5 * R + LIN * N * N))
    name=ma_n${N}_r${R}
    [ "$LIN" = 1 ] && name=${name}_lin
    build_net "$name" "$nc" "$HERE/plugins/mass_action_gold.c" "-DMA_N=$N -DMA_R=$R -DMA_LINEAR=$LIN"
done
echo "build_ref.sh: built $(ls "$OUT"/*.so | wc -l) libraries in $OUT"
