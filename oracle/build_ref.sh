#!/usr/bin/env bash
# Builds the reference simulator's own CPU engine (and, when the product's
# drop-in libraries exist, the reference CLIs linked against them) into
# oracle/_ref/.  Test infrastructure only: the product never links anything
# built here.
#
#   oracle/_ref/libref_f32.so   unmodified reference core (FP32) + kernel_stub
#                               + oracle/ref_harness.cpp
#   oracle/_ref/libref_f64.so   the same core after a scripted FP64 widening
#                               (float complex -> double complex, crealf/
#                               cimagf/cpowf -> creal/cimag/cpow, float
#                               accumulators -> double)
#   oracle/_ref/general_ref_{f32,f64}.out, grover_ref_{f32,f64}.out,
#   oracle/_ref/shor_ref_{f32,f64}.out
#                               the reference CLIs on the stub GPU backend
#   oracle/_ref/general_b200_{f32,f64}.out, grover_b200_{f32,f64}.out,
#   oracle/_ref/shor_b200_{f32,f64}.out,
#   oracle/_ref/libref_dropin_{f32,f64}.so
#                               the same reference objects with the GPU
#                               backend replaced at link time by
#                               libhgm_dropin_{f32,f64}.so (only when those
#                               exist)
#   oracle/_ref/libref_gpu_f32.so, {general,grover,shor}_refgpu_f32.out
#                               the unmodified FP32 core and CLIs with the
#                               reference's own GPU backend (src/core/kernel.cu)
#                               compiled for sm_100a (one scripted fix, see below)
#
# Sources are read where they lie under the reference tree, whose root the
# caller names in REF_ROOT (required; nothing is built without it); the widened copy is written to a scratch folder
# under oracle/_ref/ and removed after compilation.  Compiler flags follow
# the reference makefile (makefile:33,92): -O3 -fopenmp -fcx-limited-range
# on the four engine files, default flags elsewhere; -fPIC is added so the
# objects can go into a shared library.
set -euo pipefail

HERE="$(cd "$(dirname "$0")" && pwd)"
REPO="$(cd "$HERE/.." && pwd)"
REF_ROOT="${REF_ROOT:-}"
OUT="$HERE/_ref"
DROPIN_DIR="$REPO/simulador_quantico_b200/lib"

if [ -z "$REF_ROOT" ]; then
    echo "build_ref.sh: REF_ROOT (the reference tree's root) is not set; keeping existing oracle/_ref" >&2
    exit 0
fi
if [ ! -d "$REF_ROOT/src/core" ]; then
    echo "build_ref.sh: reference tree not found at $REF_ROOT; keeping existing oracle/_ref" >&2
    exit 0
fi

mkdir -p "$OUT"
CXX="${REF_CXX:-g++}"
ENGINE_FILES="dgm_core dgm_parser dgm_cpu_exec dgm_par_exec"
PLAIN_FILES="common gates lib_general lib_grover lib_shor lib_shor_number_theory lib_shor_circuits cli_common kernel_stub"

build_variant() {
    local prec="$1"        # f32 | f64
    local real="$2"        # float | double
    local work="$OUT/work_$prec"
    rm -rf "$work"
    mkdir -p "$work/src" "$work/include" "$work/obj"
    cp -r "$REF_ROOT/src/." "$work/src/"
    cp -r "$REF_ROOT/include/." "$work/include/"
    if [ "$prec" = "f64" ]; then
        find "$work/src" "$work/include" -type f \( -name '*.cpp' -o -name '*.h' \) -print0 |
            xargs -0 sed -i -E \
                -e 's/\bfloat\b/double/g' \
                -e 's/\bcrealf\b/creal/g' \
                -e 's/\bcimagf\b/cimag/g' \
                -e 's/\bcpowf\b/cpow/g'
    fi
    local inc="-I$work/include"
    for f in $ENGINE_FILES; do
        local src
        src="$(find "$work/src" -name "$f.cpp" | head -1)"
        $CXX $inc -fPIC -fopenmp -O3 -fcx-limited-range -c "$src" -o "$work/obj/$f.o"
    done
    for f in $PLAIN_FILES; do
        local src
        src="$(find "$work/src" -name "$f.cpp" | head -1)"
        $CXX $inc -fPIC -c "$src" -o "$work/obj/$f.o"
    done
    $CXX $inc -fPIC -fopenmp -c "$work/src/cli/general.cpp" -o "$work/obj/general.o"
    $CXX $inc -fPIC -fopenmp -c "$work/src/cli/grover.cpp" -o "$work/obj/grover.o"
    $CXX $inc -fPIC -fopenmp -c "$work/src/cli/shor.cpp" -o "$work/obj/shor.o"
    $CXX $inc -I"$work/include" -DREF_REAL="$real" -fPIC -O2 -fopenmp \
        -c "$HERE/ref_harness.cpp" -o "$work/obj/ref_harness.o"

    local core=""
    for f in dgm_core dgm_parser dgm_cpu_exec dgm_par_exec common gates lib_general lib_grover lib_shor \
             lib_shor_number_theory lib_shor_circuits cli_common; do
        core="$core $work/obj/$f.o"
    done
    $CXX -shared -o "$OUT/libref_$prec.so" $core "$work/obj/kernel_stub.o" "$work/obj/ref_harness.o" -fopenmp
    $CXX -o "$OUT/general_ref_$prec.out" "$work/obj/general.o" $core "$work/obj/kernel_stub.o" -fopenmp
    $CXX -o "$OUT/grover_ref_$prec.out" "$work/obj/grover.o" $core "$work/obj/kernel_stub.o" -fopenmp
    $CXX -o "$OUT/shor_ref_$prec.out" "$work/obj/shor.o" $core "$work/obj/kernel_stub.o" -fopenmp

    # The reference's own GPU backend (makefile:49-59, GPU=real), FP32 only
    # (kernel.cu is written for cuFloatComplex), compiled for sm_100a with the
    # makefile's kernel flags (makefile:26,93) and one scripted change:
    # GpuExecution01 declares max_target_bit uninitialised (kernel.cu:206) and
    # reads it at :235 when a batch holds only targets below coalesced_bits,
    # so region_start_bit -- and every address of that launch -- would come
    # from an indeterminate value.  It is initialised to 0 here, which keeps
    # such a batch at region_start_bit = coalesced_bits, inside the state.
    if [ "$prec" = "f32" ] && command -v "${NVCC:-nvcc}" > /dev/null; then
        sed -i 's/int max_target_bit, min_target_bit = coalesced_bits;/int max_target_bit = 0, min_target_bit = coalesced_bits;/' \
            "$work/src/core/kernel.cu"
        grep -q "int max_target_bit = 0, min_target_bit" "$work/src/core/kernel.cu" || {
            echo "build_ref.sh: kernel.cu patch did not apply" >&2
            exit 1
        }
        "${NVCC:-nvcc}" -arch=sm_100a -O3 -D OPS_BLOCK=300 -Xcompiler -fPIC $inc -c "$work/src/core/kernel.cu" \
            -o "$work/obj/kernel.o"
        "${NVCC:-nvcc}" -arch=sm_100a -shared -o "$OUT/libref_gpu_$prec.so" $core "$work/obj/kernel.o" \
            "$work/obj/ref_harness.o" -Xcompiler -fopenmp
        for cli in general grover shor; do
            "${NVCC:-nvcc}" -arch=sm_100a -o "$OUT/${cli}_refgpu_$prec.out" "$work/obj/$cli.o" $core \
                "$work/obj/kernel.o" -Xcompiler -fopenmp
        done
    fi

    # Link-time replacement of the GPU backend (makefile:51-61) by the
    # product's drop-in library, when it has been built.
    local dropin="$DROPIN_DIR/libhgm_dropin_$prec.so"
    if [ -f "$dropin" ]; then
        local rp="-Wl,-rpath,\$ORIGIN/../../simulador_quantico_b200/lib"
        $CXX -shared -o "$OUT/libref_dropin_$prec.so" $core "$work/obj/ref_harness.o" \
            -L"$DROPIN_DIR" -lhgm_dropin_$prec $rp -fopenmp
        $CXX -o "$OUT/general_b200_$prec.out" "$work/obj/general.o" $core \
            -L"$DROPIN_DIR" -lhgm_dropin_$prec $rp -fopenmp
        $CXX -o "$OUT/grover_b200_$prec.out" "$work/obj/grover.o" $core \
            -L"$DROPIN_DIR" -lhgm_dropin_$prec $rp -fopenmp
        $CXX -o "$OUT/shor_b200_$prec.out" "$work/obj/shor.o" $core \
            -L"$DROPIN_DIR" -lhgm_dropin_$prec $rp -fopenmp
    fi
    rm -rf "$work"
}

build_variant f32 float
build_variant f64 double
echo "build_ref.sh: built $(ls "$OUT" | tr '\n' ' ')"
