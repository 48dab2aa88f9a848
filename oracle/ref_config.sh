#!/bin/sh
# Test infrastructure (oracle). Writes a configured copy of the reference's
# config.h for one compile-time variant into oracle/_ref/<variant>/cfg/.
# The reference selects problem, grid size and adiabatic index at compile time
# (config.h:29 WHICHPROBLEM, config.h:355-362 NB_*/BS_*, config.h:107 GAMMA),
# so every grid size the host build is checked on needs its own config.
#
# fixup_cell (GPU_fixup.h:989-1006) has no return statement once its floor
# body is compiled out (#if 0), so a host compiler may assume its radius test
# `r < radfix_dens` always passes and return garbage. The configured copy ends
# the test with `return 0;`, the evident intent: floors off, no failure flag.
#
# With PLAIN=1 in the environment the radfix_dens line is left as written:
# that copy serves the host build of the CPU fixup.c, whose fixup1zone uses
# the macro as a plain constant.
#
# usage: ref_config.sh <refdir> <outdir> <mode: torus|cart> <BS_1> <BS_2> <BS_3> <gamma-expr> [opts]
#   opts: comma-separated build switches; mc = linear MC reconstruction (PPM 0),
#         hllc = HLLC Riemann solver (HLLC 1, which turns on FRAME_TRANSFORM),
#         hlld = HLLD Riemann solver (HLLD 1, likewise)
set -e
REF="$1"; OUT="$2"; MODE="$3"; B1="$4"; B2="$5"; B3="$6"; GAM="$7"; OPTS="${8:-}"
mkdir -p "$OUT"
RADFIX='s/^#define radfix_dens 0.0[[:space:]]*$/#define radfix_dens 0.0) { pf[RHO] = 1.0; pf[UU] = 0.1; } return 0; if (0/'
[ -n "${PLAIN:-}" ] && RADFIX='s/^$//'
sed -e 's/^#define WHICHPROBLEM .*/#define WHICHPROBLEM TORUS_PROBLEM/' \
    -e "s|^#define GAMMA[[:space:]].*|#define GAMMA ($GAM)|" \
    -e 's/^#define NB_1 .*/#define NB_1 1/' \
    -e 's/^#define NB_2 .*/#define NB_2 1/' \
    -e 's/^#define NB_3 .*/#define NB_3 1/' \
    -e "s/^#define BS_1 .*/#define BS_1 $B1/" \
    -e "s/^#define BS_2 .*/#define BS_2 $B2/" \
    -e "s/^#define BS_3 .*/#define BS_3 $B3/" \
    -e 's/^#define SCUDA .*/#define SCUDA (0)/' \
    -e "$RADFIX" \
    "$REF/config.h" > "$OUT/config.h.tmp"
if [ "$MODE" = "cart" ]; then
  sed -i -e 's/^#define CARTESIAN (0)/#define CARTESIAN (1)/' \
         -e 's/^#define SPHERICAL_GR (1)/#define SPHERICAL_GR (0)/' "$OUT/config.h.tmp"
fi
case ",$OPTS," in
  *,mc,*) sed -i -e 's/^#define PPM (1)/#define PPM (0)/' "$OUT/config.h.tmp" ;;
esac
case ",$OPTS," in
  *,hllc,*) sed -i -e 's/^#define HLLC (0)/#define HLLC (1)/' "$OUT/config.h.tmp" ;;
esac
case ",$OPTS," in
  *,hlld,*) sed -i -e 's/^#define HLLD (0)/#define HLLD (1)/' "$OUT/config.h.tmp" ;;
esac
mv "$OUT/config.h.tmp" "$OUT/config.h"
