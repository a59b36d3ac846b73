# Builds the C restatement of the reference hot path twice: FP32 storage
# (bit-faithful to the reference CPU solver) and FP64 storage (the FP64
# oracle).  Test infrastructure only.
OUT ?= oracle/_build
CC  ?= gcc
CFLAGS := -O2 -fPIC -std=c11 -ffp-contract=off -Wall -Wextra -Wno-unused-parameter

all: $(OUT)/liboracle_f32.so $(OUT)/liboracle_f64.so

$(OUT)/liboracle_f32.so: oracle/nimbus_oracle.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -shared -DREAL=float $< -o $@ -lm

$(OUT)/liboracle_f64.so: oracle/nimbus_oracle.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -shared -DREAL=double -DORACLE_FP64 $< -o $@ -lm

.PHONY: all
