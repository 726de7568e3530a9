#!/bin/bash
# Batch driver for the MultiQW drop-in, with the reference's run.sh contract
# (run.sh:1-40): the same two arguments, the same n and m lists and the same
# split of the problems into <number_of_threads> contiguous ranges, each run
# as its own MultiQW process in the background (run.sh:27-38).
#
# One difference, on purpose: the reference's processes all append to
# ./output_<n>_<m>, so the file holds the ranges in completion order. Here
# every range runs in its own scratch directory, and once all of an (n, m)
# pass have finished their results are appended to ./output_<n>_<m> in range
# order — the file lists the problems in index order, deterministically, the
# same bytes as one MultiQW run over the whole range. Per-range stdout is
# printed in range order too. A failing range stops the driver with status 1
# before anything of that (n, m) pass is appended.
#
# Environment (all optional):
#   MQW_N_VALUES   n values, default "5 6"   (run.sh:13)
#   MQW_M_VALUES   m values, default "1 2"   (run.sh:14)
#   MQW_PROBLEMS   problems per file, default 2000 (run.sh:27-28)
#   MQW_DEVICES    GPUs to deal the ranges to, round-robin, default "0"
#   MULTIQW_BIN    the MultiQW binary, default _lib/MultiQW beside this script
#   MQW_DRY_RUN=1  print the range commands instead of running them
set -u

if [ "$#" -ne 2 ]; then
    echo "Usage: $0 <number_of_threads> <filename_prefix>"
    exit 1
fi

num_threads=$1
filename_prefix=$2
if ! [[ "$num_threads" =~ ^[1-9][0-9]*$ ]]; then
    echo "number_of_threads must be a positive integer" >&2
    exit 1
fi

here=$(cd "$(dirname "$0")" && pwd)
bin=${MULTIQW_BIN:-$here/_lib/MultiQW}
read -r -a n_values <<< "${MQW_N_VALUES:-5 6}"
read -r -a m_values <<< "${MQW_M_VALUES:-1 2}"
read -r -a devices <<< "${MQW_DEVICES:-0}"
problems=${MQW_PROBLEMS:-2000}
dry=${MQW_DRY_RUN:-0}

work=$(mktemp -d)
trap 'rm -rf "$work"' EXIT

for n in "${n_values[@]}"; do
    filename="${filename_prefix}_${n}n"
    if [ ! -f "$filename" ]; then
        echo "File not found: $filename"
        continue
    fi
    file_abs=$(cd "$(dirname "$filename")" && pwd)/$(basename "$filename")

    # run.sh:27-28 and :31-32: contiguous ranges, the first `extra` one longer
    base=$((problems / num_threads))
    extra=$((problems % num_threads))

    for m in "${m_values[@]}"; do
        pids=()
        dirs=()
        for (( thread=0; thread<num_threads; thread++ )); do
            start_point=$((thread * base + (thread < extra ? thread : extra)))
            count=$((base + (thread < extra ? 1 : 0)))
            [ "$count" -gt 0 ] || continue
            dev=${devices[$((thread % ${#devices[@]}))]}
            if [ "$dry" = "1" ]; then
                echo "MQW_DEVICE=$dev $bin $n $m $file_abs $start_point $count"
                continue
            fi
            d="$work/${n}_${m}_${thread}"
            mkdir -p "$d"
            dirs+=("$d")
            ( cd "$d" && MQW_DEVICE=$dev exec "$bin" "$n" "$m" "$file_abs" "$start_point" "$count" \
                > stdout 2> stderr ) &
            pids+=($!)
        done
        [ "$dry" = "1" ] && continue
        status=0
        for pid in "${pids[@]}"; do
            wait "$pid" || status=1
        done
        if [ "$status" -ne 0 ]; then
            for d in "${dirs[@]}"; do cat "$d/stderr" >&2; done
            echo "run.sh: a range of n=$n, m=$m failed; output_${n}_${m} left unchanged" >&2
            exit 1
        fi
        for d in "${dirs[@]}"; do
            cat "$d/stdout"
            cat "$d/output_${n}_${m}" >> "output_${n}_${m}"
        done
    done
done
