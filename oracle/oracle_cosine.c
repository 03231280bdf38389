/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.  Never linked into the product library.
 *
 * The deterministic f32 cosine dissimilarity of the reference, restated:
 * evoc-rs native/fast_cosine.c:4-13 (compiled there with -O3 -ffast-math by
 * build.rs:1-10).  This translation unit is built with the same flags so
 * that the compiler is free to vectorise / reassociate the reduction in the
 * same way; `oracle/Makefile` also builds the reference's own file into
 * oracle/_ref/ and tests/test_oracle.py checks the two agree bit-for-bit.
 */
float orc_fast_cosine_fastmath(const float *x, const float *y, int dim) {
    float acc = 0.0f;
    for (int t = 0; t < dim; t++) acc += x[t] * y[t];
    if (acc > 0.0f) return -acc;
    return 1.17549435e-38f; /* f32::MIN_POSITIVE sentinel */
}
