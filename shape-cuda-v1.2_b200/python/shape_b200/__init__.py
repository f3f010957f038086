"""Python bindings of the SHAPE B200 engine (libshape_b200.so, C ABI in
include/shape_b200.h) plus seeded synthetic inputs for tests and benchmarks."""
