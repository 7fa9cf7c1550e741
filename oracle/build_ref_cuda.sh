#!/bin/bash
# Build the reference's own CUDA program for sm_100, for three cases, into
# oracle/_ref/.  TEST INFRASTRUCTURE: the binaries are the reference solver
# itself, used as a parity pin and as the reference GPU baseline; nothing in
# the product links or calls them.
#
#   REF=<reference checkout> bash oracle/build_ref_cuda.sh
#
# The reference tree is copied to a scratch folder under /tmp and only that
# copy is edited (the reference stays read-only):
#   - src/var.h            BC_PROBLEM selects the case
#   - src/saveData.cu      gets #include <cstring> (it uses std::memcpy without it)
#   - case constants.inc / output.inc: grid size, Re, steps, binary output on
# Outputs (git-ignored, travel with the repository snapshot):
#   _ref/refsim_lid64        lidDrivenCavity_3D, D3Q19, 64^3, Re 100, lid 0.05, N_STEPS from argv-free constant
#   _ref/refsim_tgv256_q27   taylorGreen, D3Q27, 256^3, Re 1600, u0 0.04, 1000 steps
#   _ref/refsim_bench256     benchmark (README table case), D3Q19, 256^3, 1000 steps
#   _ref/refsim_lid64_edges  C1 with the lid's edges typed as edge walls
#   _ref/refsim_lid16_trace  16^3 lid cavity writing its fields after every step
#   _ref/refsim_rb64         rayleighBenard_Periodic (thermal), 64 x 64 x 8, 1000 steps
#   _ref/cases/*             the same cases compiled in this library's case mode
#   _ref/refsim_voxel64      voxel (sphere.csv obstacle), D3Q19, 64^3, 500 steps
#   _ref/refsim_bingham32    Bingham channel, D3Q19, 32 x 32 x 64, Re 10, 1000 steps
#   _ref/refsim_lid64_ckpt   C1 (edges as walls), 1000 steps, checkpoint after step 500
#   _ref/refsim_lid64_load   C1 (edges as walls) to step 1000 from a checkpoint
# CASES_ONLY=1 rebuilds only the case-mode programs; THERMAL_ONLY=1 only refsim_rb64;
# VOXEL_ONLY=1 only refsim_voxel64; BINGHAM_ONLY=1 only refsim_bingham32; CKPT_ONLY=1 only the
# two checkpoint programs.
set -euo pipefail
REF=${REF:?set REF to the reference checkout (its src/ folder is read)}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
mkdir -p "$OUT"
[ -d "$REF/src" ] || { echo "reference tree not found at $REF" >&2; exit 1; }

build_case() {
    local name=$1 case=$2 lattice=$3 steps=$4 n=$5 extra=$6 nvflags=${7:-}
    local work
    work=$(mktemp -d /tmp/mrlbm_refbuild.XXXXXX)
    cp -r "$REF/src" "$work/src"
    chmod -R u+w "$work/src"
    cd "$work/src"
    sed -i "s/^#define BC_PROBLEM .*/#define BC_PROBLEM $case/" var.h
    sed -i '1i #include <cstring>' saveData.cu
    local c="cases/$case"
    sed -i "s/^constexpr int N = .*/constexpr int N = $n;/" "$c/constants.inc"
    sed -i "s/^constexpr int N_STEPS = .*/constexpr int N_STEPS = $steps;/" "$c/constants.inc"
    sed -i "s/^#define D3Q[0-9]*/#define $lattice/" "$c/model.inc"
    sed -i 's/^#define BIN_SAVE .*/#define BIN_SAVE (true)/; s/^#define VTK_SAVE .*/#define VTK_SAVE (false)/; s/^#define ONLY_FINAL_MACRO .*/#define ONLY_FINAL_MACRO (true)/; s/^#define MACR_SAVE .*/#define MACR_SAVE (false)/' "$c/output.inc"
    eval "$extra"
    "$NVCC" -gencode arch=compute_100,code=sm_100 -rdc=true -O3 --restrict -DSM_100 -DTARGET_LINUX $nvflags \
        -diag-suppress=39 -diag-suppress=179 -w -ccbin /usr/bin/g++ *.cu -lcudadevrt -lcurand -o "$OUT/$name"
    cd /
    rm -rf "$work"
    echo "built $OUT/$name"
}

# which blocks run: all of them, or the one an *_ONLY variable names
ONLY="${CASES_ONLY:-}${THERMAL_ONLY:-}${VOXEL_ONLY:-}${CKPT_ONLY:-}${BINGHAM_ONLY:-}"

if [ -z "$ONLY" ]; then
# C1: lid-driven cavity 64^3, Re 100, lid velocity 0.05 (tau from Re, constants.inc:35-36)
build_case refsim_lid64 lidDrivenCavity_3D D3Q19 2000 64 \
  'sed -i "s/^constexpr dfloat RE = .*/constexpr dfloat RE = 100;/; s/^constexpr dfloat U_MAX = .*/constexpr dfloat U_MAX = 0.05;/" "$c/constants.inc"; sed -i "s/^#define REPORT_SAVE .*/#define REPORT_SAVE (false)/" "$c/output.inc"'

# C1 again, with the lid's edges and corners typed as the edge/corner wall
# types of nodeTypeMap.h (zero velocity) instead of the moving lid: then no
# node reads a population from outside the domain as known (the case as
# shipped types every y = NY-1 node NORTH, so its lid edges and corners take
# some outside populations as known, fed from the reference's ghost-face
# arrays), and the run pins the solver independently of the reference's 8^3
# ghost-block layout.  The override is appended to the case's
# bc_initialization.inc, which runs after its if/else chain.
build_case refsim_lid64_edges lidDrivenCavity_3D D3Q19 2000 64 \
  'sed -i "s/^constexpr dfloat RE = .*/constexpr dfloat RE = 100;/; s/^constexpr dfloat U_MAX = .*/constexpr dfloat U_MAX = 0.05;/" "$c/constants.inc"; sed -i "s/^#define REPORT_SAVE .*/#define REPORT_SAVE (false)/" "$c/output.inc"; printf "\nif (y == (NY - 1) && (x == 0 || x == (NX - 1) || z == 0 || z == (NZ_TOTAL - 1))) {\n    nodeType = NORTH | (x == 0 ? WEST : 0) | (x == (NX - 1) ? EAST : 0) | (z == 0 ? BACK : 0) | (z == (NZ_TOTAL - 1) ? FRONT : 0);\n}\n" >> "$c/bc_initialization.inc"'

# lid-driven cavity 16^3 with the macroscopic fields written after every step
# (MACR_SAVE 1), 20 steps: a step-by-step trace for parity debugging
build_case refsim_lid16_trace lidDrivenCavity_3D D3Q19 20 16 \
  'sed -i "s/^constexpr dfloat RE = .*/constexpr dfloat RE = 100;/; s/^constexpr dfloat U_MAX = .*/constexpr dfloat U_MAX = 0.05;/" "$c/constants.inc"; sed -i "s/^#define REPORT_SAVE .*/#define REPORT_SAVE (false)/; s/^#define MACR_SAVE .*/#define MACR_SAVE (1)/; s/^#define ONLY_FINAL_MACRO .*/#define ONLY_FINAL_MACRO (false)/" "$c/output.inc"'

# C2: Taylor-Green 256^3 D3Q27, Re 1600, u0 0.04; the 53,248-byte static shared
# array of the D3Q27 kernel is over the 48 KB static limit, so the reference's
# own DYNAMIC_SHARED_MEMORY switch is turned on (definitions.h:67, main.cu:186-195)
build_case refsim_tgv256_q27 taylorGreen D3Q27 1000 256 \
  'sed -i "s/^constexpr dfloat RE = .*/constexpr dfloat RE = 1600;/; s/^constexpr dfloat U_MAX = .*/constexpr dfloat U_MAX = 0.04;/; s/^constexpr int N_STEPS = .*/constexpr int N_STEPS = 1000;/" "$c/constants.inc"; sed -i "s|^//#define DYNAMIC_SHARED_MEMORY|#define DYNAMIC_SHARED_MEMORY|" definitions.h; sed -i "s/^#define REPORT_SAVE .*/#define REPORT_SAVE (100)/; s/^#define SAVEDATA .*/#define SAVEDATA (true)/; s/^#define BIN_SAVE .*/#define BIN_SAVE (false)/" "$c/output.inc"'

# README benchmark case, D3Q19 256^3 (the published MLUPS table), 1000 steps
build_case refsim_bench256 benchmark D3Q19 1000 256 'true'
fi

if [ -z "$ONLY" ] || [ -n "${VOXEL_ONLY:-}" ]; then
# voxel obstacle case (VOXEL_FILENAME "sphere.csv", read from the working
# directory), 64^3 periodic, 500 steps.  As shipped its U_MAX = 0 gives
# TAU = 0.5 (no viscosity) and its fluid starts at rest with the body force
# zeroed in the kernel (mlbm.cu:76-78), so nothing would move: U_MAX = 0.05
# (TAU 0.519 at RE 500) and an initial uniform flow U_0_Z = 0.02 past the
# obstacle make the run exercise the 254 voxel wall types.  Its FZ = 1e-6 is
# set to 0 (the reference's kernel drops the force; this library applies it).
build_case refsim_voxel64 voxel D3Q19 500 64 \
  'sed -i "s/^constexpr dfloat U_MAX = .*/constexpr dfloat U_MAX = 0.05;/; s/^constexpr dfloat U_0_Z = .*/constexpr dfloat U_0_Z = 0.02;/; s/^constexpr dfloat FZ = .*/constexpr dfloat FZ = 0.0;/" "$c/constants.inc"; sed -i "s/^#define REPORT_SAVE .*/#define REPORT_SAVE (false)/" "$c/output.inc"'
fi
[ -n "${VOXEL_ONLY:-}" ] && exit 0

if [ -z "$ONLY" ] || [ -n "${BINGHAM_ONLY:-}" ]; then
# Bingham channel (parallelPlates_D3Q19_turbulent_Bingham: walls in y,
# periodic x and z, body force along z, a Bingham fluid with yield stress
# S_Y = Bn U_MAX^2, a log-law start with cuRAND perturbations), shrunk from
# 192 x 192 x 1536 to 32 x 32 x 64 (del = 16, NZ = 4 del) and run at Re 10
# instead of 180 (tau 0.528 instead of 0.5015, which such a coarse grid does
# not survive), 1000 steps.  Its FZ = U_TAU^2 / del is set to 0 (the
# reference's kernel drops the force, src/mlbm.cu:76-78; this library applies
# it): the log-law start decays under the walls and the yield stress.
# The case's treat_data.inc (turbulence statistics: mean flow and velocity
# fluctuations per distance from the walls) runs at a report at step 500
# (REPORT_SAVE, MACR_SAVE 500 for its mean counter, SAVEDATA on to write its
# files).
build_case refsim_bingham32 parallelPlates_D3Q19_turbulent_Bingham D3Q19 1000 32 \
  'sed -i "s/^constexpr int del = .*/constexpr int del = 16;/; s/^constexpr unsigned int NZ = .*/constexpr unsigned int NZ = 4*del;/; s/^constexpr dfloat RE = .*/constexpr dfloat RE = 10.0;/; s/^constexpr dfloat FZ = .*/constexpr dfloat FZ = 0.0;/" "$c/constants.inc"; sed -i "s/^#define REPORT_SAVE .*/#define REPORT_SAVE (500)/; s/^#define MACR_SAVE .*/#define MACR_SAVE (500)/; s/^#define SAVEDATA .*/#define SAVEDATA (true)/" "$c/output.inc"'
fi
[ -n "${BINGHAM_ONLY:-}" ] && exit 0

if [ -z "$ONLY" ] || [ -n "${CKPT_ONLY:-}" ]; then
# checkpoint interchange, on C1 with the lid's edges as walls, 1000 steps:
# refsim_lid64_ckpt writes its checkpoint file set and its macroscopic fields
# (.bin and legacy VTK) after step 500 (CHECKPOINT_SAVE, MACR_SAVE 500);
# refsim_lid64_load starts from a checkpoint file set
# (LOAD_CHECKPOINT true: the step from the last int of
# ..\\bin\\TEST\\000\\checkpoint\\_curr_step.bin, a name the reference builds
# with Windows separators, the arrays from TEST/000/checkpoint/_*.bin)
LID_EDGES='sed -i "s/^constexpr dfloat RE = .*/constexpr dfloat RE = 100;/; s/^constexpr dfloat U_MAX = .*/constexpr dfloat U_MAX = 0.05;/" "$c/constants.inc"; sed -i "s/^#define REPORT_SAVE .*/#define REPORT_SAVE (false)/" "$c/output.inc"; printf "\nif (y == (NY - 1) && (x == 0 || x == (NX - 1) || z == 0 || z == (NZ_TOTAL - 1))) {\n    nodeType = NORTH | (x == 0 ? WEST : 0) | (x == (NX - 1) ? EAST : 0) | (z == 0 ? BACK : 0) | (z == (NZ_TOTAL - 1) ? FRONT : 0);\n}\n" >> "$c/bc_initialization.inc"'
build_case refsim_lid64_ckpt lidDrivenCavity_3D D3Q19 1000 64 \
  "$LID_EDGES"'; sed -i "s/^#define CHECKPOINT_SAVE .*/#define CHECKPOINT_SAVE 500/" "$c/constants.inc"; sed -i "s/^#define MACR_SAVE .*/#define MACR_SAVE (500)/; s/^#define VTK_SAVE .*/#define VTK_SAVE (true)/; s/^#define ONLY_FINAL_MACRO .*/#define ONLY_FINAL_MACRO (false)/" "$c/output.inc"'
build_case refsim_lid64_load lidDrivenCavity_3D D3Q19 1000 64 \
  "$LID_EDGES"'; sed -i "s/^#define LOAD_CHECKPOINT .*/#define LOAD_CHECKPOINT true/" "$c/constants.inc"'
fi
[ -n "${CKPT_ONLY:-}" ] && exit 0

if [ -z "$ONLY" ] || [ -n "${THERMAL_ONLY:-}" ]; then
# thermal: rayleighBenard_Periodic (D3Q19 flow + D3G19 scalar, THERMAL_MODEL),
# 64 x 64 x 8, Pr 10, Ra 1e5, hot WEST / cold EAST walls, gravity along x,
# 1000 steps; final rho, u and C as .bin.  The case ships NZ = 4, which is
# below the 8^3 block (NUM_BLOCK_Z = NZ / BLOCK_NZ = 0, definitions.h:107-110)
# and crashes on the host; NZ = 8 is the smallest depth the program runs.  Its
# flow_initialization.inc reads randomNumbers[] (times 0) while the case leaves
# RANDOM_NUMBERS undefined, so that buffer would never be allocated
# (main.cuh:919-929): RANDOM_NUMBERS is switched on to give the read a buffer.
# Built as the stock script builds it, the thermal step kernel needs more than
# 128 registers a thread and fails to launch with its 512-thread blocks ("too
# many resources requested"; the program then writes its initial fields), so
# this one program gets -maxrregcount=128.
build_case refsim_rb64 rayleighBenard_Periodic D3Q19 1000 64 \
  'sed -i "s/^constexpr int NZ = .*/constexpr int NZ = 8;        \/\/ size z of the grid in one GPU/" "$c/constants.inc"; sed -i "s|^//#define RANDOM_NUMBERS true|#define RANDOM_NUMBERS true|" "$c/model.inc"; sed -i "s/^#define REPORT_SAVE .*/#define REPORT_SAVE (false)/" "$c/output.inc"' \
  -maxrregcount=128
fi
[ -n "${THERMAL_ONLY:-}" ] && exit 0

# ---------------------------------------------------------------------------
# The same reference cases compiled, unchanged, in this library's case mode
# (mr-lbm_b200/casebuild.py reads the case folder and pastes its snippets into
# the sm_100a step kernel).  Test fixtures for the drop-in path: they run on the
# GPU next to the reference programs above, on identical inputs.
PY=${PY:-python}
CB="$HERE/../mr-lbm_b200/casebuild.py"
mkdir -p "$OUT/cases"
common_out='--set BIN_SAVE=(true) --set VTK_SAVE=(false) --set ONLY_FINAL_MACRO=(true) --set MACR_SAVE=(false)'
$PY "$CB" "$REF/src/cases/lidDrivenCavity_3D" -o "$OUT/cases/lid64" --set N=64 --set RE=100 --set U_MAX=0.05 \
    --set N_STEPS=2000 --set "REPORT_SAVE=(false)" $common_out
$PY "$CB" "$REF/src/cases/taylorGreen" -o "$OUT/cases/tgv256_q27" --lattice 27 --set N=256 --set RE=1600 \
    --set U_MAX=0.04 --set N_STEPS=1000 --set "REPORT_SAVE=(100)" --set "SAVEDATA=(true)" $common_out
$PY "$CB" "$REF/src/cases/benchmark" -o "$OUT/cases/bench256" --set N_STEPS=1000 $common_out
# voxel obstacle case as refsim_voxel64 runs it
$PY "$CB" "$REF/src/cases/voxel" -o "$OUT/cases/voxel64" --set N=64 --set N_STEPS=500 --set U_MAX=0.05 \
    --set U_0_Z=0.02 --set FZ=0.0 --set "REPORT_SAVE=(false)" $common_out
# Bingham channel as refsim_bingham32 runs it
$PY "$CB" "$REF/src/cases/parallelPlates_D3Q19_turbulent_Bingham" -o "$OUT/cases/bingham32" --set del=16 \
    --set NZ=4*del --set RE=10.0 --set FZ=0.0 --set N_STEPS=1000 $common_out --set "REPORT_SAVE=(500)" --set "MACR_SAVE=(500)" \
    --set "SAVEDATA=(true)"
# thermal: rayleighBenard_Periodic as refsim_rb64 runs it (NZ = 8, 1000 steps)
$PY "$CB" "$REF/src/cases/rayleighBenard_Periodic" -o "$OUT/cases/rb64" --set NZ=8 --set N_STEPS=1000 \
    --set "REPORT_SAVE=(false)" $common_out
echo "built case-mode programs in $OUT/cases"
