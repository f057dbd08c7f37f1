#!/bin/sh
# Builds the reference's own helpers and its cuFFT path from their sources (oracle/_ref/), for
# the oracle only. The reference checkout is read where this container mounts it, or from
# CDK_REFERENCE_DIR; without one (the GPU box) the prebuilt oracle/_ref files are used as they
# are and this script does nothing.
ref="${CDK_REFERENCE_DIR:-/root/reference}"
[ -d "$ref/src" ] || exit 0
exec make -s -C "$(dirname "$0")" ref REF="$ref"
