#!/bin/sh
# Test infrastructure: compiles the reference's own CPU path (SPILADY 1.0,
# `-DCPU -DOMP -DSLDHL`, as its make.sh:6 does with g++) from its unmodified
# sources, for use as a checker and as the timed CPU baseline.
#
# The reference selects its physics with #defines in control.h, which
# spilady.h:45 includes from its own directory.  So for each mode this script
# makes oracle/_ref/src_<mode>/ holding symbolic links to every reference
# .cpp/.h file except control.h and spilady.cpp (whose main() is replaced by
# oracle/ref/harness.cpp), writes that mode's control.h there, and compiles.
# No reference source is copied; all outputs stay under oracle/_ref/.
#
#   nve     NVE spin-lattice (no thermostat)
#   lang    + spinlang + lattlang        (Langevin spin and lattice)
#   langte  + eltemp + localcolmot + renormalizeEnergy
#   baro    NVE + PRESSURE + STRESS  (Berendsen barostats, scale.cpp)
#   dtstep  NVE + changestep          (adaptive time step, scale_step_CPU.cpp)
# and the other Hamiltonians (-DMD, -DSDH, -DSDHL, -DSLDH in place of -DSLDHL),
# each without thermostats and with the Langevin thermostats of its degrees
# of freedom:
#   md md_lang  sdh sdh_lang  sdhl sdhl_lang  sldh sldh_lang
# and each with the electron temperature (+ renormalizeEnergy; SLDH also
# localcolmot):
#   md_te  sdh_te  sdhl_te  sldh_te
# and SLDHL with an external field and force read from files, and with the
# quantum thermostat on the lattice:
#   extf  quant
# and NVE SLDHL whose potential's 36 constants are read from theta.in, for
# finite differences of the reference's own code in them: DD05.cpp and
# JijFe.cpp are replaced at link time by oracle/ref/param_pot.cpp, which
# restates their forms:
#   param
# and the reference's own main loop (spilady.cpp, reading variables.in and a
# configuration file), NVE SLDHL, on its CPU step functions and on the B200
# engine's (oracle/ref/core_B200.cpp linked in front of the reference's
# objects, against spilady_b200/_lib/libsld_b200.so):
#   main_nve  b200_nve
#
# usage: sh oracle/ref/build.sh [reference_dir]   (default: $SPILADY_REFERENCE,
# else the reference tree mounted at /root/reference)
set -e
REF=${1:-${SPILADY_REFERENCE:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$(cd "$HERE/.." && pwd)/_ref
if [ ! -f "$REF/core.cpp" ]; then
    echo "reference sources not found at $REF" >&2
    exit 1
fi
mkdir -p "$OUT"
# the system g++ (an inherited CXX may point at a compiler without libgomp)
CXX=${ORACLE_CXX:-g++}
BASE="-O3 -fopenmp -U_FORTIFY_SOURCE -D_FORTIFY_SOURCE=0 -DCPU -DOMP -w"

for mode in nve lang langte baro dtstep md md_lang sdh sdh_lang sdhl sdhl_lang sldh sldh_lang \
           md_te sdh_te sdhl_te sldh_te extf quant param main_nve b200_nve; do
    case "$mode" in
    md*) ham=MD ;;
    sdhl*) ham=SDHL ;;
    sdh*) ham=SDH ;;
    sldh*) ham=SLDH ;;
    *) ham=SLDHL ;;
    esac
    FLAGS="$BASE -D$ham"
    src="$OUT/src_$mode"
    obj="$OUT/obj_$mode"
    mkdir -p "$src" "$obj"
    find "$src" -maxdepth 1 -type l -delete
    for f in "$REF"/*.cpp "$REF"/*.h; do
        b=$(basename "$f")
        case "$b" in control.h) continue ;; esac
        # the reference's own main loop only in the main_* and b200_* builds
        case "$mode:$b" in main_*:spilady.cpp|b200_*:spilady.cpp) ;; *:spilady.cpp) continue ;; esac
        if [ "$mode" = param ]; then
            case "$b" in DD05.cpp|JijFe.cpp) continue ;; esac
        fi
        ln -s "$f" "$src/$b"
    done
    {
        echo "/* control.h for mode $mode, written by oracle/ref/build.sh */"
        echo "#define readconf"
        echo "#define runstep"
        case "$mode" in
        lang) echo "#define spinlang"; echo "#define lattlang" ;;
        langte)
            echo "#define spinlang"; echo "#define lattlang"
            echo "#define eltemp"; echo "#define localcolmot"
            echo "#define renormalizeEnergy" ;;
        baro) echo "#define PRESSURE"; echo "#define STRESS" ;;
        dtstep) echo "#define changestep" ;;
        md_lang) echo "#define lattlang" ;;
        sdh_lang|sdhl_lang) echo "#define spinlang" ;;
        sldh_lang) echo "#define spinlang"; echo "#define lattlang" ;;
        md_te) echo "#define lattlang"; echo "#define eltemp"; echo "#define renormalizeEnergy" ;;
        sdh_te|sdhl_te)
            echo "#define spinlang"; echo "#define eltemp"; echo "#define renormalizeEnergy" ;;
        sldh_te)
            echo "#define spinlang"; echo "#define lattlang"; echo "#define eltemp"
            echo "#define localcolmot"; echo "#define renormalizeEnergy" ;;
        extf) echo "#define extfield"; echo "#define extforce" ;;
        main_nve|b200_nve) ;;
        quant) echo "#define lattlang"; echo "#define quantumnoise" ;;
        esac
    } > "$src/control.h.new"
    if ! cmp -s "$src/control.h.new" "$src/control.h"; then
        mv "$src/control.h.new" "$src/control.h"
    else
        rm -f "$src/control.h.new"
    fi
    pids=""
    extra="$HERE/harness.cpp"
    if [ "$mode" = param ]; then extra="$extra $HERE/param_pot.cpp"; fi
    case "$mode" in
    main_*) extra="" ;;
    b200_*) extra="$HERE/core_B200.cpp" ;;
    esac
    for f in "$src"/*.cpp $extra; do
        b=$(basename "$f" .cpp)
        o="$obj/$b.o"
        if [ ! -f "$o" ] || [ "$f" -nt "$o" ] || [ "$src/control.h" -nt "$o" ]; then
            $CXX $FLAGS -I"$src" -I"$HERE/../../include" -c "$f" -o "$o" &
            pids="$pids $!"
        fi
    done
    for p in $pids; do wait "$p"; done
    case "$mode" in
    b200_*)
        # the backend's definitions first: the linker keeps the first of the
        # step functions the reference's *_CPU.cpp objects define again
        lib=$(cd "$HERE/../../spilady_b200/_lib" && pwd)
        $CXX -fopenmp "$obj/core_B200.o" $(ls "$obj"/*.o | grep -v '/core_B200\.o$') \
            -Wl,--allow-multiple-definition -L"$lib" -lsld_b200 -Wl,-rpath,'$ORIGIN/../../spilady_b200/_lib' \
            -o "$OUT/spilady_ref_$mode" -lm ;;
    *)
        $CXX -fopenmp "$obj"/*.o -o "$OUT/spilady_ref_$mode" -lm ;;
    esac
done
echo "built: $(ls "$OUT"/spilady_ref_* | tr '\n' ' ')"
