# Builds the C restatement oracle (test infrastructure only):
#   make -f oracle/oracle.mk        ->  oracle/_build/libwcoracle.so
HERE := $(dir $(lastword $(MAKEFILE_LIST)))
OUT := $(HERE)_build
CC ?= gcc
# plain IEEE double arithmetic: no fast-math, no FMA contraction
CFLAGS := -O2 -std=gnu99 -fPIC -ffp-contract=off -Wall -Wno-unused-variable

$(OUT)/libwcoracle.so: $(HERE)wc_oracle.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -shared -o $@ $< -lm
