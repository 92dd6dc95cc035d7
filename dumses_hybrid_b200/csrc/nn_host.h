// Library-internal accessors shared by the step code and the surrogate network.
#pragma once
#include "dumses_gpu.h"
#include "nn_features.cuh"

int dg_nn_view(const dg_nn *n, dg::nn::NetView *v);
int dg_nn_device(const dg_nn *n);
float *dg_nn_sample_x(dg_nn *n);
float *dg_nn_sample_t(dg_nn *n);
void dg_nn_set_count(dg_nn *n, long long c);
