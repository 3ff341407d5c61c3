#!/usr/bin/env bash
# Test infrastructure only: compiles the reference's own CUDA Recon
# (AreTomo3 AreTomo/Recon + the MaUtil/DataUtil/MrcUtil files it needs) for
# sm_100a from the reference sources where they lie, plus this directory's
# driver and stub, into oracle/_ref/ref_recon; and its projection-alignment
# re-projector (AreTomo/ProjAlign/GReproj + CCalcReproj) into
# oracle/_ref/ref_reproj; and its input stage (AreTomo/Correct/GCorrPatchShift
# + the Fourier crop of CFourierCropImage) with the thickness measurement
# (AreTomo/Recon/CCalcVolThick) into oracle/_ref/ref_stack; and its MRC volume
# writer (LibSrc/Mrcfile CSaveMrc, host C++ only) into oracle/_ref/ref_mrc.
# Nothing is copied out of the
# reference tree; objects go to oracle/_ref/obj.
set -euo pipefail
REF=${AT3R_REFERENCE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/../_ref"
OBJ="$OUT/obj"
mkdir -p "$OBJ"
[ -d "$REF/AreTomo/Recon" ] || { echo "reference tree not found at $REF: oracle/_ref not built (set AT3R_REFERENCE)" >&2; exit 0; }
NVCC=${NVCC:-nvcc}
CUFLAGS="-std=c++17 -O2 -Xptxas -dlcm=ca -gencode arch=compute_100a,code=sm_100a -I$REF/LibSrc/Include -I$REF"
CXXFLAGS="-std=c++17 -O2 -pthread -m64 -I$REF/LibSrc/Include -I$REF -I/usr/local/cuda/include"
CU="AreTomo/Recon/GBackProj AreTomo/Recon/GBackProjWbp AreTomo/Recon/GDiffProj AreTomo/Recon/GForProj
    AreTomo/Recon/GRWeight AreTomo/Recon/GWeightProjs AreTomo/Recon/GCalcRFactor
    MaUtil/GFFT1D MaUtil/GFillEmpty2D MaUtil/GGenRandoms MaUtil/GFourierResize2D MaUtil/GFFTUtil2D"
CPP="AreTomo/Recon/CTomoBase AreTomo/Recon/CTomoWbp AreTomo/Recon/CTomoSart AreTomo/Recon/CDoBaseRecon
     AreTomo/Recon/CDoWbpRecon AreTomo/Recon/CDoSartRecon MaUtil/CCufft2D MaUtil/CPad2D MaUtil/CSimpleFuncs
     AreTomo/Util/CSplitItems DataUtil/CTiltSeries DataUtil/CMrcStack AreTomo/MrcUtil/CAlignParam
     AreTomo/MrcUtil/CDarkFrames LibSrc/Mrcfile/Image/C4BitImage LibSrc/Util/Util_Time"
objs=()
for f in $CU; do
  o="$OBJ/$(echo "$f" | tr / _).o"
  [ "$o" -nt "$REF/$f.cu" ] || $NVCC $CUFLAGS -c "$REF/$f.cu" -o "$o"
  objs+=("$o")
done
for f in $CPP; do
  o="$OBJ/$(echo "$f" | tr / _).o"
  [ "$o" -nt "$REF/$f.cpp" ] || g++ $CXXFLAGS -c "$REF/$f.cpp" -o "$o"
  objs+=("$o")
done
g++ $CXXFLAGS -c "$HERE/ref_stub.cpp" -o "$OBJ/ref_stub.o"
g++ $CXXFLAGS -c "$HERE/ref_driver.cpp" -o "$OBJ/ref_driver.o"
$NVCC -gencode arch=compute_100a,code=sm_100a -o "$OUT/ref_recon" "${objs[@]}" \
  "$OBJ/ref_stub.o" "$OBJ/ref_driver.o" -lcufft -lcurand -lcuda
echo "built $OUT/ref_recon"

# the drop-in shim (integration/at3r_recon_shim.cpp: CDoWbpRecon / CDoSartRecon
# with their bodies calling libat3r) linked in place of the reference's
# CDoWbpRecon.cpp / CDoSartRecon.cpp, with the same driver: oracle/_ref/shim_recon
LIBDIR="$HERE/../../aretomo3_b200"
if [ -f "$LIBDIR/libat3r.so" ]; then
  g++ $CXXFLAGS -I"$HERE/../../include" -c "$HERE/../../integration/at3r_recon_shim.cpp" -o "$OBJ/at3r_recon_shim.o"
  sh=()
  for o in "${objs[@]}"; do
    case "$o" in *AreTomo_Recon_CDoWbpRecon.o|*AreTomo_Recon_CDoSartRecon.o) ;; *) sh+=("$o") ;; esac
  done
  $NVCC -gencode arch=compute_100a,code=sm_100a -o "$OUT/shim_recon" "${sh[@]}" "$OBJ/at3r_recon_shim.o" \
    "$OBJ/ref_stub.o" "$OBJ/ref_driver.o" -L"$LIBDIR" -lat3r -Xlinker -rpath -Xlinker '$ORIGIN/../../aretomo3_b200' \
    -lcufft -lcurand -lcuda
  echo "built $OUT/shim_recon"
fi

# the projection-alignment re-projector (AreTomo/ProjAlign/GReproj.cu + CCalcReproj.cpp)
rp=()
for f in AreTomo/ProjAlign/GReproj; do
  o="$OBJ/$(echo "$f" | tr / _).o"
  [ "$o" -nt "$REF/$f.cu" ] || $NVCC $CUFLAGS -c "$REF/$f.cu" -o "$o"
  rp+=("$o")
done
for f in AreTomo/ProjAlign/CCalcReproj; do
  o="$OBJ/$(echo "$f" | tr / _).o"
  [ "$o" -nt "$REF/$f.cpp" ] || g++ $CXXFLAGS -c "$REF/$f.cpp" -o "$o"
  rp+=("$o")
done
g++ $CXXFLAGS -c "$HERE/ref_reproj_driver.cpp" -o "$OBJ/ref_reproj_driver.o"
$NVCC -gencode arch=compute_100a,code=sm_100a -o "$OUT/ref_reproj" "${rp[@]}" "$OBJ/ref_reproj_driver.o"
echo "built $OUT/ref_reproj"

# the input stage (AreTomo/Correct/GCorrPatchShift.cu, CCorrectUtil.cpp) and the
# thickness measurement (AreTomo/Recon/CCalcVolThick.cpp) on top of the Recon objects
st=()
for f in AreTomo/Correct/GCorrPatchShift; do
  o="$OBJ/$(echo "$f" | tr / _).o"
  [ "$o" -nt "$REF/$f.cu" ] || $NVCC $CUFLAGS -c "$REF/$f.cu" -o "$o"
  st+=("$o")
done
for f in AreTomo/Correct/CCorrectUtil AreTomo/Recon/CCalcVolThick; do
  o="$OBJ/$(echo "$f" | tr / _).o"
  [ "$o" -nt "$REF/$f.cpp" ] || g++ $CXXFLAGS -c "$REF/$f.cpp" -o "$o"
  st+=("$o")
done
g++ $CXXFLAGS -c "$HERE/ref_stack_stub.cpp" -o "$OBJ/ref_stack_stub.o"
g++ $CXXFLAGS -c "$HERE/ref_stack_driver.cpp" -o "$OBJ/ref_stack_driver.o"
$NVCC -gencode arch=compute_100a,code=sm_100a -o "$OUT/ref_stack" "${objs[@]}" "${st[@]}" \
  "$OBJ/ref_stub.o" "$OBJ/ref_stack_stub.o" "$OBJ/ref_stack_driver.o" -lcufft -lcurand -lcuda
echo "built $OUT/ref_stack"

# the MRC volume writer (LibSrc/Mrcfile, host code: builds and runs without a GPU)
mr=()
for f in LibSrc/Mrcfile/App/CSaveMrc LibSrc/Mrcfile/Header/CSaveMainHeader LibSrc/Mrcfile/Header/CSaveExtHeader \
         LibSrc/Mrcfile/Header/CMainHeader LibSrc/Mrcfile/Image/CSaveImage LibSrc/Util/Util_FileName \
         LibSrc/Util/Util_SwapByte LibSrc/Util/Util_String; do
  o="$OBJ/$(echo "$f" | tr / _).o"
  [ "$o" -nt "$REF/$f.cpp" ] || g++ $CXXFLAGS -w -I"$REF/LibSrc" -c "$REF/$f.cpp" -o "$o"
  mr+=("$o")
done
g++ $CXXFLAGS -I"$REF/LibSrc" -c "$HERE/ref_mrc_driver.cpp" -o "$OBJ/ref_mrc_driver.o"
g++ -o "$OUT/ref_mrc" "${mr[@]}" "$OBJ/ref_mrc_driver.o"
echo "built $OUT/ref_mrc"
