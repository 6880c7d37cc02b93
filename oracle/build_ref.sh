#!/usr/bin/env bash
# Build the reference's own programs (comer, makedb, db2bin) for sm_100a from
# the sources where they lie in the reference tree, with nvcc/g++ directly (no
# CMake), outputs only into oracle/_ref/.  TEST INFRASTRUCTURE: the binaries
# are the reference oracle run on a B200 to pin this project's results; the
# product never calls them.
#
# usage: oracle/build_ref.sh <reference-root>
#        (or COMER2_REFERENCE=<reference-root> oracle/build_ref.sh)
set -euo pipefail
REF=${1:-${COMER2_REFERENCE:-}}
if [ -z "$REF" ] || [ ! -d "$REF/src" ]; then
    echo "usage: $0 <reference-root> (the reference's source tree, with src/)" >&2
    exit 2
fi
SRC="$REF/src"
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
OBJ="$OUT/obj"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
JOBS=${JOBS:-$(nproc)}
mkdir -p "$OBJ"

# source files named in the add_library/add_executable lists of a CMakeLists.txt
srcs() {
    python3 - "$1" <<'EOF'
import re, sys, os
d = os.path.dirname(sys.argv[1])
txt = "\n".join(ln.split("#")[0] for ln in open(sys.argv[1]).read().splitlines())
for m in re.finditer(r"add_(?:library|executable)\s*\(\s*\w+(?:\s+STATIC)?(.*?)\)", txt, re.S):
    for tok in m.group(1).split():
        if re.search(r"\.(cpp|cu|c)$", tok):
            print(os.path.join(d, tok))
EOF
}

DEFS="-DCOMERSTATEDIR=$OUT/var -DCOMER_INSTALL_DIR=$OUT"
# every library's own directory is a PUBLIC include directory in the CMake files
INC="-I$SRC -I$SRC/extsp -I$SRC/liblib -I$SRC/libseg -I$SRC/libHDP -I$SRC/libpro -I$SRC/libmycu"
CXXFLAGS="-O2 -std=c++11 -include string -pthread $DEFS $INC"
NVFLAGS="-O2 -std=c++11 -gencode arch=compute_100a,code=sm_100a -rdc=true --pre-include string -Xcompiler -pthread $DEFS $INC"

LIBS="extsp liblib libseg libHDP libpro libmycu"
compile_one() {
    local f=$1 o=$2 incdir=$3
    if [ -f "$o" ] && [ "$o" -nt "$f" ]; then return 0; fi
    case "$f" in
        *.cu) $NVCC $NVFLAGS -I"$incdir" -c "$f" -o "$o" ;;
        *.c|*.cpp) $NVCC -x cu $NVFLAGS -I"$incdir" -c "$f" -o "$o" ;;
    esac
}
export -f compile_one
export NVCC NVFLAGS CXXFLAGS

lists=""
for L in $LIBS; do
    for f in $(srcs "$SRC/$L/CMakeLists.txt"); do
        o="$OBJ/$L/$(echo "${f#$SRC/$L/}" | tr '/' '_').o"
        mkdir -p "$OBJ/$L"
        echo "$f $o $(dirname "$f")"
    done
done > "$OBJ/libsources.txt"
for P in comer makedb db2bin; do
    for f in $(srcs "$SRC/$P/CMakeLists.txt"); do
        mkdir -p "$OBJ/$P"
        echo "$f $OBJ/$P/$(basename "$f").o $(dirname "$f")"
    done
done > "$OBJ/progsources.txt"

cat "$OBJ/libsources.txt" "$OBJ/progsources.txt" | xargs -P "$JOBS" -L 1 bash -c 'compile_one "$0" "$1" "$2"'

LIBOBJS=$(awk '{print $2}' "$OBJ/libsources.txt" | tr '\n' ' ')
for P in comer makedb db2bin; do
    POBJS=$(awk -v p="$OBJ/$P/" 'index($2, p) == 1 {print $2}' "$OBJ/progsources.txt" | tr '\n' ' ')
    $NVCC -gencode arch=compute_100a,code=sm_100a -rdc=true -o "$OUT/$P" $POBJS $LIBOBJS -lcudadevrt -lpthread
done
# parameter files the programs read at start-up (COMERSTATEDIR)
mkdir -p "$OUT/var"
cp "$SRC/env/comer.par" "$SRC/env/ssss" "$SRC/env/cvs2s" "$OUT/var/"
sed 's/^\s*SCOADJ\s*=.*/SCOADJ = no/' "$SRC/env/options.txt" > "$OUT/var/options.txt"
echo "built: $OUT/comer $OUT/makedb $OUT/db2bin"
