// Namespace of the kernel headers. Every translation unit compiles them into
// `vb` except vb_stage_f64c.cu, which defines VB_NS before its includes to get
// a second FP64 instantiation of the stage kernels, built with FMA
// contraction, under names of its own.
#pragma once
#ifndef VB_NS
#define VB_NS vb
#endif
