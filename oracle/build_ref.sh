#!/bin/bash
# Builds the oracle's reference-derived libraries into oracle/_ref from the
# reference sources where they lie (read-only; nothing is copied):
#   libref_walk.so   reference tree build + P2P list walk (src/fmm.c, src/operator.c,
#                    src/global.c, src/memory.c, src/utility.cc) + oracle/ref_walk_harness.c
#                    + oracle/ref_entry_record.c (records the lists)
#   libref_pair.so   reference pair arithmetic (src/gpu_kernel.impl.h) host-compiled
#                    in three variants (FP64, FP64+GPUCUTOFF, FP32 SPI+GPUCUTOFF)
#   libref_dropin_{dp,sp,act}.so reference walk + harness + the B200 drop-in gpu_entry
#                    (photons-on-mt3000_b200/csrc/gpu_entry_b200.cpp) + the multi-pack
#                    harness oracle/ref_pack_harness.c, linked to libphotons_p2p.so;
#                    built only when that library exists (act: the FP64 form built
#                    with ACT_OPT, the reference's active-level sink filter).
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $PHOTONS_REFERENCE, else /root/reference.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REPO="$(cd "$HERE/.." && pwd)"
REF="${1:-${PHOTONS_REFERENCE:-/root/reference}}"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
if [ ! -f "$REF/src/fmm.c" ]; then
  echo "build_ref: reference sources not found at $REF; keeping prebuilt oracle/_ref" >&2
  exit 0
fi
mkdir -p "$OBJ"
CFLAGS="-O2 -fPIC -fopenmp -I$HERE/ref_shim -I$REF/inc -DLONGSHORT -DPERIODIC_CONDITION -DGPUP2P -DCPU_DP -w"
for f in fmm operator global memory; do
  gcc $CFLAGS -c "$REF/src/$f.c" -o "$OBJ/$f.o"
done
g++ $CFLAGS -include cstdio -c "$REF/src/utility.cc" -o "$OBJ/utility.o"
gcc $CFLAGS -c "$HERE/ref_walk_harness.c" -o "$OBJ/ref_walk_harness.o"
gcc $CFLAGS -c "$HERE/ref_entry_record.c" -o "$OBJ/ref_entry_record.o"
WALK_OBJS="$OBJ/fmm.o $OBJ/operator.o $OBJ/global.o $OBJ/memory.o $OBJ/utility.o $OBJ/ref_walk_harness.o"
g++ -shared -fopenmp -Wl,-Bsymbolic -o "$OUT/libref_walk.so" $WALK_OBJS "$OBJ/ref_entry_record.o"

# FP64 variants pin oracle/p2p_oracle.c bit for bit: both are built without
# FMA contraction. The FP32 SPI variant is the timed CPU baseline: vectorised
# for the host (AVX2 + FMA), as a production host build would be.
PFLAGS="-O2 -fPIC -fopenmp -ffp-contract=off -I$HERE/ref_shim -I$REF/src -w"
g++ $PFLAGS -DGPU_DP -DREF_SUFFIX=dp -c "$HERE/ref_pair.cpp" -o "$OBJ/ref_pair_dp.o"
g++ $PFLAGS -DGPU_DP -DGPUCUTOFF -DREF_SUFFIX=dp_cut -c "$HERE/ref_pair.cpp" -o "$OBJ/ref_pair_dp_cut.o"
g++ -O3 -fPIC -fopenmp -march=x86-64-v3 -I$HERE/ref_shim -I$REF/src -w -DSPI -DGPUCUTOFF -DREF_SUFFIX=sp_spi \
  -c "$HERE/ref_pair.cpp" -o "$OBJ/ref_pair_sp_spi.o"
g++ -shared -fopenmp -o "$OUT/libref_pair.so" "$OBJ/ref_pair_dp.o" "$OBJ/ref_pair_dp_cut.o" "$OBJ/ref_pair_sp_spi.o"

PKG="$REPO/photons-on-mt3000_b200"
if [ -f "$PKG/photons_p2p/libphotons_p2p.so" ]; then
  g++ $CFLAGS -std=c++17 -I"$REPO/include" -DGPU_DP -DGPUCUTOFF -c "$PKG/csrc/gpu_entry_b200.cpp" -o "$OBJ/gpu_entry_b200_dp.o"
  g++ $CFLAGS -std=c++17 -I"$REPO/include" -DGPUCUTOFF -c "$PKG/csrc/gpu_entry_b200.cpp" -o "$OBJ/gpu_entry_b200_sp.o"
  g++ $CFLAGS -std=c++17 -I"$REPO/include" -DGPU_DP -DGPUCUTOFF -DACT_OPT -c "$PKG/csrc/gpu_entry_b200.cpp" \
    -o "$OBJ/gpu_entry_b200_act.o"
  gcc $CFLAGS -c "$HERE/ref_pack_harness.c" -o "$OBJ/ref_pack_harness.o"
  for v in dp sp act; do
    g++ -shared -fopenmp -Wl,-Bsymbolic -o "$OUT/libref_dropin_$v.so" $WALK_OBJS "$OBJ/ref_pack_harness.o" "$OBJ/gpu_entry_b200_$v.o" \
      -L"$PKG/photons_p2p" -lphotons_p2p -Wl,-rpath,'$ORIGIN/../../photons-on-mt3000_b200/photons_p2p'
  done
fi
# The drop-in over a host stand-in for the pass protocol (oracle/host_session_stub.c):
# CPU tests of the drop-in's host logic; no CUDA library involved.
g++ $CFLAGS -std=c++17 -I"$REPO/include" -DGPUCUTOFF -c "$PKG/csrc/gpu_entry_b200.cpp" -o "$OBJ/gpu_entry_b200_host.o"
g++ $CFLAGS -std=c++17 -I"$REPO/include" -DGPUCUTOFF -DACT_OPT -c "$PKG/csrc/gpu_entry_b200.cpp" \
  -o "$OBJ/gpu_entry_b200_hostact.o"
gcc $CFLAGS -I"$REPO/include" -c "$HERE/host_session_stub.c" -o "$OBJ/host_session_stub.o"
[ -f "$OBJ/ref_pack_harness.o" ] || gcc $CFLAGS -c "$HERE/ref_pack_harness.c" -o "$OBJ/ref_pack_harness.o"
for v in host hostact; do
  g++ -shared -fopenmp -Wl,-Bsymbolic -o "$OUT/libref_dropin_$v.so" $WALK_OBJS "$OBJ/ref_pack_harness.o" \
    "$OBJ/gpu_entry_b200_$v.o" "$OBJ/host_session_stub.o"
done
rm -rf "$OBJ"
echo "build_ref: built $(ls "$OUT" | tr '\n' ' ')"
