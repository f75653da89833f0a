# AutoRIFTGPU: the Julia side of libautorift_gpu's C ABI (include/autorift_gpu.h).
#
# A drop-in for AutoRIFT.jl's correlator with the reference's own types (ImagePair, PointSet,
# Params, DisplacementField, MultichipResult), computed on a B200 through `ccall`: `track!`,
# `correlate_multichip`, the three `autorift` forms and the `init` / `reinit!` / `autorift!`
# cache lifecycle, plus `submit` for the request loop. The FFI idiom is the reference's FFTW
# binding (src/plans.jl:271-312): a `const` library path, raw `Ptr{Cvoid}` handles (one
# context per device, cached under a `ReentrantLock`), no finalizers, and a non-zero status
# turned into a Julia exception naming the failure.
#
# Device memory: a `Cache` owns its prepared pair on the device until `close(cache)` (or the
# next `reinit!`, which replaces it); every other call uploads what it needs and frees it
# before returning. Nothing is cached globally except the per-device context.
#
# Load after AutoRIFT:
#     using AutoRIFT; include("AutoRIFTGPU.jl"); using .AutoRIFTGPU
#     out = AutoRIFTGPU.track(pair, pts, p)          # same result type as AutoRIFT.track
#     cache = AutoRIFTGPU.init(a, b; grid_spacing = 8)
#     r = AutoRIFTGPU.autorift!(cache)               # MultichipResult
#     AutoRIFTGPU.reinit!(cache; secondary = c); r2 = AutoRIFTGPU.autorift!(cache)
#     close(cache)

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

# A pair resident on the device (`ar_pair`). Owned by whoever made it; `release!` frees it.
mutable struct DevicePair
    handle::Ptr{Cvoid}
    ctx::Ptr{Cvoid}
end

function release!(dp::DevicePair)
    if dp.handle != C_NULL
        ccall((:ar_pair_destroy, LIB), Cint, (Ptr{Cvoid},), dp.handle)
        dp.handle = C_NULL
    end
    return nothing
end

# Upload a host pair (ar_pair_upload). The library copies the arrays out before returning.
function upload(pair::ImagePair, ctx::Ptr{Cvoid})
    T = eltype(pair.reference)
    ref = collect(pair.reference)          # dense column-major copies (no-ops for Matrix)
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
    return DevicePair(h[], ctx)
end

# Run `f(dp)` on a temporary device copy of `pair`, freed afterwards.
function with_device(f, pair::ImagePair, ctx::Ptr{Cvoid})
    dp = upload(pair, ctx)
    try
        return f(dp)
    finally
        release!(dp)
    end
end

"""
    AutoRIFTGPU.track!(out, pair, pts, p; subpixel = p.subpixel, measure = first(p.similarity))

`AutoRIFT.track!` (src/track.jl:103-152) on the GPU: same arguments, same semantics, same
`DisplacementField` written in place. `pair` is a host `ImagePair` (uploaded for the call) or a
`DevicePair` already on the device.
"""
function track!(out::DisplacementField, pair::ImagePair, pts::PointSet, p::Params;
                device::Integer = 0, kw...)
    ctx = context(device)
    with_device(dp -> track!(out, dp, pts, p; kw...), pair, ctx)
end

function track!(out::DisplacementField, dp::DevicePair, pts::PointSet, p::Params;
                subpixel = p.subpixel, measure = first(p.similarity))
    length(out) == length(pts) || throw(DimensionMismatch(
        "output has $(length(out)) points but the point set has $(length(pts))"))
    ctx = dp.ctx
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

track(pair::Union{ImagePair,DevicePair}, pts::PointSet, p::Params; kw...) =
    track!(displacement_field(pts), pair, pts, p; kw...)

prepare_opts(m::NoPreprocess, q) = ArPrepareOpts(AR_PRE_NONE, 0, 0.0, quant_code(q))
prepare_opts(m::Highpass, q) = ArPrepareOpts(AR_PRE_HIGHPASS, m.width, 0.0, quant_code(q))
prepare_opts(m::Wallis, q) = ArPrepareOpts(AR_PRE_WALLIS, m.width, m.min_std, quant_code(q))
prepare_opts(m, q) = throw(ArgumentError("$(typeof(m)) has no GPU implementation"))
quant_code(::QuantizeUInt8) = AR_QUANT_UINT8
quant_code(::NoQuantize) = AR_QUANT_NONE

# `_prepare` (src/api.jl:305-311) on the device: the raw pair is uploaded, filtered and
# quantised into a new device pair, and the raw copy freed. The result stays on the device.
function device_prepare(raw::ImagePair, p::Params, ctx::Ptr{Cvoid})
    opts = Ref(prepare_opts(p.preprocess, p.quantize))
    with_device(raw, ctx) do dp
        h = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:ar_prepare, LIB), Cint,
                   (Ptr{Cvoid}, Ptr{Cvoid}, Ref{ArPrepareOpts}, Ref{Ptr{Cvoid}}),
                   ctx, dp.handle, opts, h)
        check(ctx, rc, "ar_prepare")
        DevicePair(h[], ctx)
    end
end

# A device pair's images and masks as a host ImagePair of its element type.
function download(dp::DevicePair)
    ctx = dp.ctx
    dt = Ref{Cint}(0); nr = Ref{Int64}(0); nc = Ref{Int64}(0)
    check(ctx, ccall((:ar_pair_info, LIB), Cint,
                     (Ptr{Cvoid}, Ref{Cint}, Ref{Int64}, Ref{Int64}), dp.handle, dt, nr, nc),
          "ar_pair_info")
    T = dt[] == AR_U8 ? UInt8 : dt[] == AR_F32 ? Float32 : dt[] == AR_U16 ? UInt16 : Int16
    r = Matrix{T}(undef, nr[], nc[]); s = similar(r)
    rv = Matrix{Bool}(undef, nr[], nc[]); sv = similar(rv)
    rc = ccall((:ar_pair_download, LIB), Cint,
               (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Bool}, Ptr{Bool}),
               ctx, dp.handle, r, s, rv, sv)
    check(ctx, rc, "ar_pair_download")
    return ImagePair(r, s, rv, sv)
end

"""
    AutoRIFTGPU.prepare(pair, p) -> ImagePair

`_prepare` (src/api.jl:305-311) on the GPU: preprocess then quantize each image, returned as a
host `ImagePair` of the correlation element type with the filtered masks. (The pipeline itself
never takes this round trip: `init` and `autorift` keep the prepared pair on the device.)
"""
function prepare(pair::ImagePair, p::Params; device::Integer = 0)
    dp = device_prepare(pair, p, context(device))
    try
        return download(dp)
    finally
        release!(dp)
    end
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
    AutoRIFTGPU.correlate_multichip(prepared, grid::PointSet{2}, p) -> MultichipResult

`correlate_multichip` (src/multichip.jl:106-137) on the GPU, over a prepared pair: a host
`ImagePair` (uploaded for the call) or a `DevicePair` already on the device.
"""
function correlate_multichip(prepared::ImagePair, grid::PointSet, p::Params; device::Integer = 0)
    with_device(dp -> correlate_multichip(dp, grid, p), prepared, context(device))
end

function correlate_multichip(dp::DevicePair, grid::PointSet, p::Params)
    ctx = dp.ctx
    gr, gc = size(grid)
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

# The grid when the caller gives none (`_build_grid`, src/api.jl:339-347).
build_grid(imagesize, p::Params) =
    gridpoints(imagesize, p.grid_spacing; chip_size = p.chip_size_max,
               chip_aspect = p.chip_aspect, search_radius_x = p.search_radius_x,
               search_radius_y = p.search_radius_y, dx_prior = p.dx_prior,
               dy_prior = p.dy_prior)

"""
    AutoRIFTGPU.Cache

`AutoRIFT.Cache` (src/api.jl:30-44) with the prepared pair resident on the device: the
resolved parameters, the pair as supplied (`raw`, host arrays), the prepared pair (a
`DevicePair` owned by the cache), the grid, the last result and the dirty flag. Built by
`init`, advanced by `reinit!`, run by `autorift!`; `close(cache)` frees its device memory.
Not thread-safe: one cache per task, as in the reference.
"""
mutable struct Cache{P<:Params}
    params::P
    raw::ImagePair
    prepared::DevicePair
    grid::PointSet{2}
    result::Union{Nothing,MultichipResult}
    isfresh::Bool
end

"""
    AutoRIFTGPU.init(reference, secondary; reference_valid, secondary_valid, device, kw...) -> Cache

`init` (src/api.jl:66-76): resolve the keywords, filter and quantise both images on the device
(the prepared pair stays there), build the grid.
"""
function init(reference::AbstractMatrix, secondary::AbstractMatrix;
              reference_valid = nothing, secondary_valid = nothing, device::Integer = 0, kw...)
    p = AutoRIFT.params(; kw...)
    raw = ImagePair(reference, secondary; reference_valid, secondary_valid)
    prepared = device_prepare(raw, p, context(device))
    grid = build_grid(size(raw.reference), p)
    return Cache{typeof(p)}(p, raw, prepared, grid, nothing, true)
end

# The mask the cache holds for `img` (in either slot), or `nothing` (src/api.jl:325-328).
maskfor(img, old::ImagePair) =
    img === old.reference ? old.reference_valid :
    img === old.secondary ? old.secondary_valid : nothing

"""
    AutoRIFTGPU.reinit!(cache; reference, secondary, reference_valid, secondary_valid) -> cache

`reinit!` (src/api.jl:104-134): point the cache at a new pair of the same size. An omitted
image keeps its value; an omitted mask follows its image (kept only when the cache holds that
same image, matched by identity in either slot, else derived from finiteness). When nothing
changed identity the prepared pair is kept; otherwise the new pair is prepared on the device and
the old prepared pair freed. (The reference re-filters only the image that changed; the device
prepares both in a fraction of a millisecond, with the same result.)
"""
function reinit!(cache::Cache; reference = nothing, secondary = nothing,
                 reference_valid = nothing, secondary_valid = nothing)
    isnothing(reference) && isnothing(secondary) &&
        isnothing(reference_valid) && isnothing(secondary_valid) && return cache
    old = cache.raw
    ref = isnothing(reference) ? old.reference : reference
    sec = isnothing(secondary) ? old.secondary : secondary
    rv = isnothing(reference_valid) ? maskfor(ref, old) : reference_valid
    sv = isnothing(secondary_valid) ? maskfor(sec, old) : secondary_valid
    size(ref) == size(old.reference) && size(sec) == size(old.reference) ||
        throw(DimensionMismatch(
            "new images are $(size(ref)) and $(size(sec)) but the cache was built for " *
            "$(size(old.reference)); the grid and output arrays are sized to that. Build a " *
            "new cache with `init` for a different image size."))
    raw = ImagePair(ref, sec; reference_valid = rv, secondary_valid = sv)
    same = raw.reference === old.reference && raw.secondary === old.secondary &&
           raw.reference_valid === old.reference_valid &&
           raw.secondary_valid === old.secondary_valid
    if !same
        prepared = device_prepare(raw, cache.params, cache.prepared.ctx)
        release!(cache.prepared)
        cache.prepared = prepared
    end
    cache.raw = raw
    cache.isfresh |= true
    cache.result = nothing
    return cache
end

"""
    AutoRIFTGPU.autorift!(cache) -> MultichipResult

`autorift!` (src/api.jl:165-170): correlate the cache's current pair on the device; calling
it again before the next `reinit!` returns the same result without recomputing.
"""
function autorift!(cache::Cache)
    cache.isfresh || isnothing(cache.result) || return cache.result
    cache.result = correlate_multichip(cache.prepared, cache.grid, cache.params)
    cache.isfresh = false
    return cache.result
end

"""
    AutoRIFTGPU.imagepair(cache) -> ImagePair

The pair the correlator sees (`imagepair`, src/api.jl:52), copied back from the device.
"""
imagepair(cache::Cache) = download(cache.prepared)

"""
    close(cache)

Free the cache's prepared pair on the device. The cache cannot run again afterwards.
"""
Base.close(cache::Cache) = release!(cache.prepared)

"""
    AutoRIFTGPU.autorift(image1, image2; kw...) -> MultichipResult
    AutoRIFTGPU.autorift(image1, image2, p::Params) -> MultichipResult
    AutoRIFTGPU.autorift(image1, image2, grid::PointSet; kw...) -> MultichipResult or DisplacementField

The three forms of `autorift` (src/api.jl:210-274) on the GPU. The keyword form is
`autorift!(init(...))` with the cache closed afterwards; a gridded `PointSet{2}` runs the
multi-chip-size search over it, a scattered `PointSet{1}` runs one scale with `track`.
"""
function autorift(image1::AbstractMatrix, image2::AbstractMatrix; kw...)
    cache = init(image1, image2; kw...)
    try
        return autorift!(cache)
    finally
        close(cache)
    end
end

function autorift(image1::AbstractMatrix, image2::AbstractMatrix, p::Params; device::Integer = 0)
    dp = device_prepare(ImagePair(image1, image2), p, context(device))
    try
        return correlate_multichip(dp, build_grid(size(image1), p), p)
    finally
        release!(dp)
    end
end

function autorift(image1::AbstractMatrix, image2::AbstractMatrix, grid::PointSet;
                  reference_valid = nothing, secondary_valid = nothing, device::Integer = 0,
                  kw...)
    p = AutoRIFT.params(; kw...)
    raw = ImagePair(image1, image2; reference_valid, secondary_valid)
    dp = device_prepare(raw, p, context(device))
    try
        return run_points(dp, grid, p)
    finally
        release!(dp)
    end
end

# Dispatch on the point set's dimensionality (`_run`, src/api.jl:273-274).
run_points(dp::DevicePair, grid::PointSet{2}, p::Params) = correlate_multichip(dp, grid, p)
run_points(dp::DevicePair, pts::PointSet{1}, p::Params) = track(dp, pts, p)

# A queued request and everything it references (kept alive until it completes).
mutable struct Ticket
    ctx::Ptr{Cvoid}
    id::Int64
    keep::Any
    result::MultichipResult
end

"""
    AutoRIFTGPU.submit(image1, image2, grid, p; reference_valid, secondary_valid) -> Ticket

Queue `autorift` on the context's request loop (`ar_submit`); requests submitted from several
tasks run concurrently on the device. `fetch(ticket)` waits and returns the MultichipResult.
Masks default to all-valid for integer images and to finiteness for float images, as
`ImagePair`'s default.
"""
function submit(image1::AbstractMatrix{T}, image2::AbstractMatrix{T}, grid::PointSet, p::Params;
                reference_valid = nothing, secondary_valid = nothing,
                device::Integer = 0) where {T}
    ctx = context(device)
    ref = collect(image1); sec = collect(image2)
    rv = reference_valid === nothing ? nothing : collect(Bool, reference_valid)  # one byte per pixel
    sv = secondary_valid === nothing ? nothing : collect(Bool, secondary_valid)
    gr, gc = size(grid)
    res = MultichipResult(Matrix{Float32}(undef, gr, gc), Matrix{Float32}(undef, gr, gc),
                          Matrix{Float32}(undef, gr, gc), Matrix{UInt16}(undef, gr, gc),
                          falses(gr, gc))
    it = Matrix{UInt8}(undef, gr, gc)
    P, cols = flat_points(grid)
    Pref = Ref(P)
    angs = rotation_angles(p.rotation)  # copied by ar_submit
    req = Ref(ArRequest(pointer(ref), pointer(sec),
                        rv === nothing ? C_NULL : Ptr{UInt8}(pointer(rv)),
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
    return Ticket(ctx, t[], (ref, sec, rv, sv, cols, Pref, req, it), res)
end

function Base.fetch(t::Ticket)
    rc = ccall((:ar_wait, LIB), Cint, (Ptr{Cvoid}, Int64, Cint), t.ctx, t.id, -1)
    check(t.ctx, rc, "ar_wait")
    t.result.interpolated .= t.keep[end] .!= 0
    ccall((:ar_release, LIB), Cint, (Ptr{Cvoid}, Int64), t.ctx, t.id)
    return t.result
end

end # module
