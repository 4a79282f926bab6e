#!/bin/sh
# check_qualified.sh ORIGINAL QUALIFIED -- fails unless the two files differ
# only by the qualifier macros (and the ROUND constant of the 30-round
# PageRank build), and unless ip_compute and ip_combine were qualified.
set -e
orig="$1"; qual="$2"
grep -q '^IP_DEVICE void ip_compute(' "$qual" || { echo "ip_compute not qualified in $orig"; exit 1; }
grep -q '^IP_DEVICE void ip_combine(' "$qual" || { echo "ip_combine not qualified in $orig"; exit 1; }
# Remove the macros and the ROUND change: what is left must equal the original.
sed -e 's/^IP_DEVICE //' -e 's/^IP_GLOBAL //' -e 's/ROUND = 30;/ROUND = 10;/' "$qual" | cmp -s - "$orig" || {
    echo "qualified source of $orig differs by more than the qualifier macros"; exit 1; }
