// compact_schemes/numerics_pc.hpp -- drop-in numerics_pc<Type>
// (src/numerics_pc.hpp, src/numerics_base.hpp) over libcompact_b200.
// Type = double (full API) or float (deriv1d/deriv2d on periodic faces use
// the single-rank self halo).  The MPI exchange becomes a device copy: the
// block is its own neighbour on every interface axis.
#pragma once

#include <type_traits>

#include "common.hpp"

template <typename Type>
struct numerics_pc {
    static_assert(std::is_same<Type, double>::value || std::is_same<Type, float>::value,
                  "numerics_pc<Type>: double or float");

    numerics_pc(t_dcomp dcomp_info, int nbc[2][3]) {
        compact_b200::check(cs_numerics_create(&handle, compact_b200::to_c(dcomp_info), nbc),
                            "numerics_pc");
        compact_b200::check(cs_get_ndf(handle, ndf_), "cs_get_ndf");
        for (int f = 0; f < 2; ++f)
            for (int a = 0; a < 3; ++a) ndf[f][a] = (unsigned)ndf_[f][a];
        for (int a = 0; a < 3; ++a) {
            double *d, *s, *r;
            compact_b200::check(cs_get_buffers(handle, a, &d, &s, &r), "cs_get_buffers");
            drva_buffer[a] = d;
            send_buffer[a] = s;
            recv_buffer[a] = r;
        }
    }
    ~numerics_pc() {
        if (pbco) cudaFree(pbco);
        if (pbci) cudaFree(pbci);
        cs_numerics_destroy(handle);
    }
    numerics_pc(const numerics_pc &) = delete;
    numerics_pc &operator=(const numerics_pc &) = delete;

    // numerics_base::deriv_setup (src/numerics_base.hpp:182-297).
    void deriv_setup() {
        compact_b200::check(cs_deriv_setup(handle), "deriv_setup");
        double co[16], ci[16];
        compact_b200::check(cs_get_coeffs(handle, co, ci), "cs_get_coeffs");
        Type tco[16], tci[16];
        for (int i = 0; i < 16; ++i) { tco[i] = (Type)co[i]; tci[i] = (Type)ci[i]; }
        if (!pbco) cudaMalloc(&pbco, 16 * sizeof(Type));
        if (!pbci) cudaMalloc(&pbci, 16 * sizeof(Type));
        cudaMemcpy(pbco, tco, sizeof tco, cudaMemcpyHostToDevice);
        cudaMemcpy(pbci, tci, sizeof tci, cudaMemcpyHostToDevice);
    }

    // numerics_pc::deriv1d<Axis> (src/numerics_pc.hpp:74-119), synchronous
    // like the reference's launch.
    template <unsigned int Axis>
    void deriv1d(Type *infield, Type *outfield, int nstart, int nend, t_dcomp dcomp_info,
                 unsigned int variable_id) {
        static_assert(Axis < 3, "Axis index must be 0, 1, or 2");
        launch(Axis, infield, outfield, nstart, nend, dcomp_info, variable_id, 0, 0, nullptr);
        compact_b200::check(cudaDeviceSynchronize() == cudaSuccess ? CS_OK : CS_ERR_CUDA, "deriv1d");
    }

    // numerics_pc::deriv2d<Axis> (src/numerics_pc.hpp:121-168): component ->
    // slot Axis, asynchronous on *stream.
    template <unsigned int Axis>
    void deriv2d(Type *infield, Type *outfield, int nstart, int nend, t_dcomp dcomp_info,
                 unsigned int variable_id, unsigned int component_id, cudaStream_t *stream) {
        static_assert(Axis < 3, "Axis index must be 0, 1, or 2");
        launch(Axis, infield, outfield, nstart, nend, dcomp_info, variable_id, component_id, Axis,
               stream ? *stream : nullptr);
    }

    // numerics_pc::fill_buffers<min,max> (src/numerics_pc.hpp:231-287).
    template <unsigned int min_value, unsigned int max_value>
    void fill_buffers(Type *infield, int nrt, t_dcomp dcomp_info, cudaStream_t *streams) {
        static_assert(std::is_same<Type, double>::value,
                      "fill_buffers: FP64 fields (the interface exchange buffers are FP64; numerics_pc<float> "
                      "derivatives use the single-rank periodic closure without them)");
        compact_b200::check(cs_fill_buffers(handle, infield, min_value, max_value, nrt,
                                            compact_b200::to_c(dcomp_info), streams ? streams[0] : nullptr),
                            "fill_buffers");
    }

    // numerics_base::mpigo (src/numerics_base.hpp:119-180), single rank.
    template <typename StreamType, typename SyncFunction>
    void mpigo(t_dcomp, int[2][3], int, unsigned int variable_id, StreamType *stream, SyncFunction sync) {
        compact_b200::check(cs_halo_exchange_self(handle, variable_id, stream ? (void *)*stream : nullptr),
                            "mpigo");
        sync(stream);
    }

    cs_numerics *handle = nullptr;
    Type *drva_buffer[3];
    Type *send_buffer[3];
    Type *recv_buffer[3];
    Type *pbco = nullptr, *pbci = nullptr;
    unsigned int ndf[NumberOfFaces][NumberOfSpatialDims];

protected:
    void launch(unsigned axis, Type *in, Type *out, int nstart, int nend, t_dcomp d, unsigned var,
                unsigned comp, unsigned slot, cudaStream_t st) {
        int rc;
        if (std::is_same<Type, double>::value)
            rc = cs_deriv(handle, (int)axis, (const double *)in, (double *)out, nstart, nend,
                          compact_b200::to_c(d), var, comp, slot, CS_HALO_RECV, st);
        else
            rc = cs_deriv_f32(handle, (int)axis, (const float *)in, (float *)out, nstart, nend,
                              compact_b200::to_c(d), var, comp, slot, CS_HALO_SELF, st);
        compact_b200::check(rc, "deriv");
    }
    int ndf_[2][3];
};

// numerics_rtc<Type> (src/numerics_rtc.hpp): same kernels; the NVRTC compile
// steps are no-ops (everything is compiled ahead of time for sm_100a) and the
// face flags come from ndf as the compiled NSTART/NEND macros did.
template <typename Type>
struct numerics_rtc : public numerics_pc<Type> {
    using numerics_pc<Type>::numerics_pc;
    template <unsigned int Axis>
    void deriv1d_compile(t_dcomp, int, int) {}
    template <unsigned int Axis>
    void deriv2d_compile(t_dcomp, int, int) {}
    template <unsigned int Axis, unsigned int FaceId>
    void fill_buffer_compile() {}
    template <unsigned int Axis>
    void deriv1d(Type *infield, Type *outfield, t_dcomp d, unsigned int variable_id, cudaStream_t *stream) {
        this->launch(Axis, infield, outfield, (int)this->ndf[0][Axis], (int)this->ndf[1][Axis], d,
                     variable_id, 0, 0, stream ? *stream : nullptr);
        cudaStreamSynchronize(stream ? *stream : nullptr);
    }
    template <unsigned int Axis>
    void deriv2d(Type *infield, Type *outfield, t_dcomp d, unsigned int variable_id,
                 unsigned int component_id, cudaStream_t *stream) {
        numerics_pc<Type>::template deriv2d<Axis>(infield, outfield, (int)this->ndf[0][Axis],
                                                   (int)this->ndf[1][Axis], d, variable_id, component_id,
                                                   stream);
    }
};
