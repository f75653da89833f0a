# AutoRIFTGPU: the Julia side of libautorift_gpu's C ABI (include/autorift_gpu.h).
#
# A drop-in for AutoRIFT.jl's correlator: `track!` and `prepare` with the reference's own types
# (ImagePair, PointSet, Params, DisplacementField), computed on a B200 through `ccall`. The FFI
# idiom is the reference's FFTW binding (src/plans.jl:271-312): a `const` library path, raw
# `Ptr{Cvoid}` handles cached under a `ReentrantLock`, no finalizers on the hot path, and a
# non-zero status turned into a Julia exception naming the failure.
#
# Load after AutoRIFT:
#     using AutoRIFT; include("AutoRIFTGPU.jl"); using .AutoRIFTGPU
#     out = AutoRIFTGPU.track(pair, pts, p)          # same result type as AutoRIFT.track

module AutoRIFTGPU

using AutoRIFT
using AutoRIFT: ImagePair, PointSet, Params, DisplacementField, displacement_field,
                ZNCC, NCC, NoRefine, PyramidRefine, upsampling, scatter,
                Highpass, Wallis, NoPreprocess, QuantizeUInt8, NoQuantize,
                GardnerFilter, NoOutlierFilter, MultichipResult, gridpoints,
                RotationSearch, NoRotationSearch

const LIB = get(ENV, "AUTORIFT_GPU_LIB", joinpath(@__DIR__, "..", "libautorift_gpu.so"))

const AR_OK = Cint(0)
const AR_U8, AR_U16, AR_F32, AR_I16 = Cint(0), Cint(1), Cint(2), Cint(3)
const AR_ZNCC, AR_NCC = Cint(0), Cint(1)
const AR_PRE_NONE, AR_PRE_HIGHPASS, AR_PRE_WALLIS = Cint(0), Cint(1), Cint(2)
const AR_QUANT_NONE, AR_QUANT_UINT8 = Cint(0), Cint(1)

# `ar_points` (include/autorift_gpu.h): the eight PointSet fields, flattened, and the count.
struct ArPoints
    x::Ptr{Float64}
    y::Ptr{Float64}
    radius_x::Ptr{Int64}
    radius_y::Ptr{Int64}
    dx_prior::Ptr{Float64}
    dy_prior::Ptr{Float64}
    chip_size_x::Ptr{Int64}
    chip_size_y::Ptr{Int64}
    n::Int64
end

struct ArPrepareOpts
    preprocess::Cint
    width::Cint
    min_std::Float64
    quantize::Cint
end

# `ar_multichip_params`: the Params fields correlate_multichip reads (src/types.jl:781-829).
struct ArMultichipParams
    chip_size_base::Cint
    chip_size_min::Cint
    chip_size_max::Cint
    chip_aspect::Float64
    min_search_radius::Cint
    coarse_stride::Cint
    coarse_buffer::Cint
    min_coarse_valid_fraction::Float64
    upsampling::Cint
    measure::Cint
    outliers::Cint
    outlier_window::Cint
    outlier_iterations::Cint
    min_agree_fraction::Float64
    agree_tolerance::Float64
    mad_scale::Float64
    fill_window::Cint
    rotation_count::Cint              # 0: NoRotationSearch
    rotation_angles::Ptr{Float64}     # AutoRIFT.angles(p.rotation), read during the call
    level_measure_count::Cint         # 0: `measure` at every level
    level_measures::NTuple{8,Cint}    # measure_at(p, k) for a `similarity` tuple
end

# The chip rotations of a rotation method (src/types.jl:577), as the C ABI takes them.
rotation_angles(::NoRotationSearch) = Float64[]
rotation_angles(m::RotationSearch) = collect(Float64, AutoRIFT.angles(m))

# `ar_request`: one queued autorift() request.
struct ArRequest
    reference::Ptr{Cvoid}
    secondary::Ptr{Cvoid}
    reference_valid::Ptr{UInt8}
    secondary_valid::Ptr{UInt8}
    nrows::Int64
    ncols::Int64
    dtype::Cint
    prepare::ArPrepareOpts
    params::ArMultichipParams
    grid::Ptr{ArPoints}
    grid_rows::Int64
    grid_cols::Int64
    dx::Ptr{Float32}
    dy::Ptr{Float32}
    correlation::Ptr{Float32}
    chip_size::Ptr{UInt16}
    interpolated::Ptr{UInt8}
end

# One context per device, created on first use (the plan cache's role, src/plans.jl:25-47).
const CTX_LOCK = ReentrantLock()
const CTXS = Dict{Int,Ptr{Cvoid}}()

function context(device::Integer = 0)
    lock(CTX_LOCK) do
        get!(CTXS, Int(device)) do
            h = Ref{Ptr{Cvoid}}(C_NULL)
            rc = ccall((:ar_ctx_create, LIB), Cint, (Cint, Ref{Ptr{Cvoid}}), device, h)
            rc == AR_OK || error("ar_ctx_create($device) failed ($rc): no usable CUDA device")
            h[]
        end
    end
end

function check(ctx::Ptr{Cvoid}, rc::Cint, what::AbstractString)
    rc == AR_OK && return nothing
    buf = Vector{UInt8}(undef, 512)
    ccall((:ar_last_error, LIB), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Csize_t), ctx, buf, length(buf))
    msg = unsafe_string(pointer(buf))
    rc == 2 && throw(DimensionMismatch("$what: $msg"))
    rc == 1 && throw(ArgumentError("$what: $msg"))
    error("$what failed ($rc): $msg")
end

eltype_code(::Type{UInt8}) = AR_U8
eltype_code(::Type{UInt16}) = AR_U16
eltype_code(::Type{Int16}) = AR_I16
eltype_code(::Type{Float32}) = AR_F32
eltype_code(T::Type) = throw(ArgumentError(
    "element type $T has no GPU correlator; use UInt8, UInt16, Int16 or Float32"))

measure_code(::ZNCC) = AR_ZNCC
measure_code(::NCC) = AR_NCC
measure_code(m) = throw(ArgumentError("$(typeof(m)) has no GPU implementation"))

# A device-resident pair, keyed on the identity of the arrays it was made from: the same
# `===` reuse the reference's Cache makes (src/api.jl:325-335).
mutable struct DevicePair
    handle::Ptr{Cvoid}
    ctx::Ptr{Cvoid}
end

const PAIR_LOCK = ReentrantLock()
const PAIRS = IdDict{Any,DevicePair}()

function upload(pair::ImagePair, ctx::Ptr{Cvoid})
    key = (pair.reference, pair.secondary, pair.reference_valid, pair.secondary_valid)
    lock(PAIR_LOCK) do
        get!(PAIRS, key) do
            T = eltype(pair.reference)
            ref = collect(pair.reference)          # dense column-major copies
            sec = collect(pair.secondary)
            rv = collect(pair.reference_valid)     # Matrix{Bool}: one byte per pixel
            sv = collect(pair.secondary_valid)
            h = Ref{Ptr{Cvoid}}(C_NULL)
            nr, nc = size(ref)
            rc = ccall((:ar_pair_upload, LIB), Cint,
                       (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{UInt8}, Ptr{UInt8}, Int64,
                        Int64, Cint, Ref{Ptr{Cvoid}}),
                       ctx, ref, sec, rv, sv, nr, nc, eltype_code(T), h)
            check(ctx, rc, "ar_pair_upload")
            DevicePair(h[], ctx)
        end
    end
end

"""
    AutoRIFTGPU.track!(out, pair, pts, p; subpixel = p.subpixel, measure = first(p.similarity))

`AutoRIFT.track!` (src/track.jl:103-152) on the GPU: same arguments, same semantics, same
`DisplacementField` written in place.
"""
function track!(out::DisplacementField, pair::ImagePair, pts::PointSet, p::Params;
                subpixel = p.subpixel, measure = first(p.similarity), device::Integer = 0)
    length(out) == length(pts) || throw(DimensionMismatch(
        "output has $(length(out)) points but the point set has $(length(pts))"))
    ctx = context(device)
    dp = upload(pair, ctx)
    flat = scatter(pts)
    x, y = collect(flat.x), collect(flat.y)
    rx, ry = collect(flat.radius_x), collect(flat.radius_y)
    dx0, dy0 = collect(flat.dx_prior), collect(flat.dy_prior)
    csx, csy = collect(flat.chip_size_x), collect(flat.chip_size_y)
    n = length(x)
    dx = Vector{Float32}(undef, n)
    dy = Vector{Float32}(undef, n)
    cc = Vector{Float32}(undef, n)
    sr = Vector{UInt8}(undef, n)
    angs = rotation_angles(p.rotation)  # _correlate_rotations! (src/track.jl:313-409)
    GC.@preserve x y rx ry dx0 dy0 csx csy angs begin
        P = Ref(ArPoints(pointer(x), pointer(y), pointer(rx), pointer(ry), pointer(dx0),
                         pointer(dy0), pointer(csx), pointer(csy), n))
        rc = ccall((:ar_track_rotated, LIB), Cint,
                   (Ptr{Cvoid}, Ptr{Cvoid}, Ref{ArPoints}, Cint, Cint, Ptr{Float64}, Cint,
                    Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{UInt8}),
                   ctx, dp.handle, P, upsampling(subpixel), measure_code(measure), angs,
                   length(angs), dx, dy, cc, sr)
        check(ctx, rc, "ar_track_rotated")
    end
    vec(out.dx) .= dx
    vec(out.dy) .= dy
    vec(out.correlation) .= cc
    vec(out.searched) .= sr .!= 0
    return out
end

track(pair::ImagePair, pts::PointSet, p::Params; kw...) =
    track!(displacement_field(pts), pair, pts, p; kw...)

prepare_opts(m::NoPreprocess, q) = ArPrepareOpts(AR_PRE_NONE, 0, 0.0, quant_code(q))
prepare_opts(m::Highpass, q) = ArPrepareOpts(AR_PRE_HIGHPASS, m.width, 0.0, quant_code(q))
prepare_opts(m::Wallis, q) = ArPrepareOpts(AR_PRE_WALLIS, m.width, m.min_std, quant_code(q))
prepare_opts(m, q) = throw(ArgumentError("$(typeof(m)) has no GPU implementation"))
quant_code(::QuantizeUInt8) = AR_QUANT_UINT8
quant_code(::NoQuantize) = AR_QUANT_NONE

"""
    AutoRIFTGPU.prepare(pair, p) -> ImagePair

`_prepare` (src/api.jl:305-311) on the GPU: preprocess then quantize each image, returned as a
host `ImagePair` of the correlation element type with the filtered masks.
"""
function prepare(pair::ImagePair, p::Params; device::Integer = 0)
    ctx = context(device)
    dp = upload(pair, ctx)
    opts = Ref(prepare_opts(p.preprocess, p.quantize))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:ar_prepare, LIB), Cint,
               (Ptr{Cvoid}, Ptr{Cvoid}, Ref{ArPrepareOpts}, Ref{Ptr{Cvoid}}), ctx, dp.handle, opts, h)
    check(ctx, rc, "ar_prepare")
    dt = Ref{Cint}(0); nr = Ref{Int64}(0); nc = Ref{Int64}(0)
    check(ctx, ccall((:ar_pair_info, LIB), Cint,
                     (Ptr{Cvoid}, Ref{Cint}, Ref{Int64}, Ref{Int64}), h[], dt, nr, nc), "ar_pair_info")
    T = dt[] == AR_U8 ? UInt8 : dt[] == AR_F32 ? Float32 : dt[] == AR_U16 ? UInt16 : Int16
    r = Matrix{T}(undef, nr[], nc[]); s = similar(r)
    rv = Matrix{Bool}(undef, nr[], nc[]); sv = similar(rv)
    rc = ccall((:ar_pair_download, LIB), Cint,
               (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Bool}, Ptr{Bool}),
               ctx, h[], r, s, rv, sv)
    ccall((:ar_pair_destroy, LIB), Cint, (Ptr{Cvoid},), h[])
    check(ctx, rc, "ar_pair_download")
    return ImagePair(r, s, rv, sv)
end


outlier_fields(f::GardnerFilter) = (Cint(1), f.window, f.iterations, f.min_agree_fraction,
                                    f.agree_tolerance, f.mad_scale)
outlier_fields(::NoOutlierFilter) = (Cint(0), 5, 3, 8 / 25, 0.2, 4.0)

# `angs` = rotation_angles(p.rotation), preserved by the caller for the duration of the call.
function multichip_params(p::Params, angs::Vector{Float64})
    o = outlier_fields(p.outliers)
    ArMultichipParams(p.chip_size_base, p.chip_size_min, p.chip_size_max, p.chip_aspect,
                      p.min_search_radius, p.coarse_stride, p.coarse_buffer,
                      p.min_coarse_valid_fraction, upsampling(p.subpixel),
                      measure_code(first(p.similarity)), o[1], o[2], o[3], o[4], o[5], o[6],
                      p.fill_window, length(angs), isempty(angs) ? C_NULL : pointer(angs),
                      length(p.similarity) > 1 ? length(p.similarity) : 0,
                      ntuple(k -> measure_code(p.similarity[min(k, length(p.similarity))]), 8))
end

# The eight PointSet fields flattened, kept alive by the returned tuple.
function flat_points(pts::PointSet)
    f = scatter(pts)
    cols = (collect(f.x), collect(f.y), collect(f.radius_x), collect(f.radius_y),
            collect(f.dx_prior), collect(f.dy_prior), collect(f.chip_size_x),
            collect(f.chip_size_y))
    P = ArPoints(pointer(cols[1]), pointer(cols[2]), pointer(cols[3]), pointer(cols[4]),
                 pointer(cols[5]), pointer(cols[6]), pointer(cols[7]), pointer(cols[8]),
                 length(cols[1]))
    return P, cols
end

"""
    AutoRIFTGPU.correlate_multichip(prepared::ImagePair, grid::PointSet{2}, p) -> MultichipResult

`correlate_multichip` (src/multichip.jl:106-137) on the GPU, over a prepared pair.
"""
function correlate_multichip(prepared::ImagePair, grid::PointSet, p::Params; device::Integer = 0)
    ctx = context(device)
    dp = upload(prepared, ctx)
    gr, gc = size(grid)
    n = gr * gc
    dx = Matrix{Float32}(undef, gr, gc); dy = similar(dx); cc = similar(dx)
    cs = Matrix{UInt16}(undef, gr, gc); it = Matrix{UInt8}(undef, gr, gc)
    P, cols = flat_points(grid)
    angs = rotation_angles(p.rotation)
    prm = Ref(multichip_params(p, angs))
    GC.@preserve cols angs begin
        rc = ccall((:ar_multichip, LIB), Cint,
                   (Ptr{Cvoid}, Ptr{Cvoid}, Ref{ArPoints}, Int64, Int64, Ref{ArMultichipParams},
                    Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{UInt16}, Ptr{UInt8}),
                   ctx, dp.handle, Ref(P), gr, gc, prm, dx, dy, cc, cs, it)
        check(ctx, rc, "ar_multichip")
    end
    return MultichipResult(dx, dy, cc, cs, BitMatrix(it .!= 0))
end

"""
    AutoRIFTGPU.autorift(image1, image2; kw...) -> MultichipResult

`autorift` (src/api.jl:210-274) with the default grid: prepare both images, then the
multi-chip-size search, on the GPU.
"""
function autorift(image1::AbstractMatrix, image2::AbstractMatrix; reference_valid = nothing,
                  secondary_valid = nothing, device::Integer = 0, kw...)
    p = AutoRIFT.params(; kw...)
    pair = reference_valid === nothing && secondary_valid === nothing ? ImagePair(image1, image2) :
           ImagePair(image1, image2, something(reference_valid, isfinite.(image1)),
                     something(secondary_valid, isfinite.(image2)))
    grid = gridpoints(size(image1), p.grid_spacing; chip_size = p.chip_size_max,
                      chip_aspect = p.chip_aspect, search_radius_x = p.search_radius_x,
                      search_radius_y = p.search_radius_y, dx_prior = p.dx_prior,
                      dy_prior = p.dy_prior)
    return correlate_multichip(prepare(pair, p; device), grid, p; device)
end

# A queued request and everything it references (kept alive until it completes).
mutable struct Ticket
    ctx::Ptr{Cvoid}
    id::Int64
    keep::Any
    result::MultichipResult
end

"""
    AutoRIFTGPU.submit(image1, image2, grid, p) -> Ticket

Queue `autorift` on the context's request loop (`ar_submit`); requests submitted from several
tasks run concurrently on the device. `fetch(ticket)` waits and returns the MultichipResult.
"""
function submit(image1::AbstractMatrix{T}, image2::AbstractMatrix{T}, grid::PointSet, p::Params;
                secondary_valid = nothing, device::Integer = 0) where {T}
    ctx = context(device)
    ref = collect(image1); sec = collect(image2)
    sv = secondary_valid === nothing ? nothing : collect(secondary_valid)  # Matrix{Bool}
    gr, gc = size(grid)
    res = MultichipResult(Matrix{Float32}(undef, gr, gc), Matrix{Float32}(undef, gr, gc),
                          Matrix{Float32}(undef, gr, gc), Matrix{UInt16}(undef, gr, gc),
                          falses(gr, gc))
    it = Matrix{UInt8}(undef, gr, gc)
    P, cols = flat_points(grid)
    Pref = Ref(P)
    angs = rotation_angles(p.rotation)  # copied by ar_submit
    req = Ref(ArRequest(pointer(ref), pointer(sec), C_NULL,
                        sv === nothing ? C_NULL : Ptr{UInt8}(pointer(sv)),
                        size(ref, 1), size(ref, 2), eltype_code(T),
                        prepare_opts(p.preprocess, p.quantize), multichip_params(p, angs),
                        Base.unsafe_convert(Ptr{ArPoints}, Pref), gr, gc,
                        pointer(res.dx), pointer(res.dy), pointer(res.correlation),
                        pointer(res.chip_size), pointer(it)))
    t = Ref{Int64}(0)
    rc = GC.@preserve angs ccall((:ar_submit, LIB), Cint, (Ptr{Cvoid}, Ref{ArRequest}, Ref{Int64}),
                                 ctx, req, t)
    check(ctx, rc, "ar_submit")
    return Ticket(ctx, t[], (ref, sec, sv, cols, Pref, req, it), res)
end

function Base.fetch(t::Ticket)
    rc = ccall((:ar_wait, LIB), Cint, (Ptr{Cvoid}, Int64, Cint), t.ctx, t.id, -1)
    check(t.ctx, rc, "ar_wait")
    t.result.interpolated .= t.keep[end] .!= 0
    ccall((:ar_release, LIB), Cint, (Ptr{Cvoid}, Int64), t.ctx, t.id)
    return t.result
end

end # module
