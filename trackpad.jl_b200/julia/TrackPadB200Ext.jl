"""
    TrackPadB200Ext

Package extension of TrackPad.jl that runs `linepass!` / `ringpass!` on a B200
through libtrackpad_b200.so (C ABI: include/trackpad_b200.h).  It adds methods
for device arrays (`CuMatrix{Float64}` coordinates, `CuVector{Int}` flags) and a
`B200()` backend tag for host arrays; the CPU methods of TrackPad are untouched.

Registration in TrackPad's Project.toml (beside TrackPadCUDAExt):
    [weakdeps]    CUDA = "052768ef-5323-5732-b1bb-66c8b64840ba"
    [extensions]  TrackPadB200Ext = "CUDA"
and set ENV["TRACKPAD_B200_LIB"] to the path of libtrackpad_b200.so.
"""
module TrackPadB200Ext

using TrackPad
using TrackPad: Lattice, Beam, AbstractElement, TimeVaryingElement, TimeContext, materialize, beti
using CUDA

const LIB = get(ENV, "TRACKPAD_B200_LIB", "libtrackpad_b200.so")

# --- C structs (field order and types as in include/trackpad_b200.h) ---------
struct TpElem
    kind::Int32; max_order::Int32; num_int_steps::Int32
    fringe_bend_entrance::Int32; fringe_bend_exit::Int32; misalign_index::Int32
    iparam::NTuple{2,Int32}
    L::Float64; k::Float64; angle::Float64; e1::Float64; e2::Float64
    fint1::Float64; fint2::Float64; gap::Float64; gk::Float64
    polynom_a::NTuple{4,Float64}; polynom_b::NTuple{4,Float64}; kick_angle::NTuple{2,Float64}
    volt::Float64; freq::Float64; h::Float64; lag::Float64; philag::Float64; energy::Float64
    param::NTuple{8,Float64}
end

struct TpMisalign
    t1::NTuple{6,Float64}; t2::NTuple{6,Float64}; r1::NTuple{36,Float64}; r2::NTuple{36,Float64}
end

struct TpOpts
    size::Int32; exact_hamiltonian::Int32; device_pointers::Int32; fp_contract::Int32
    block_size::Int32; min_blocks::Int32; schedule::Int32; table_in_smem::Int32
    aperture_x::Float64; aperture_y::Float64; stream::Ptr{Cvoid}
    bounds_check::Int32; reserved0::Int32
end

struct TpLossSpec
    kind::Int32; reserved::Int32; sigma::Float64; lost_weight::Float64
end

const TP_KIND = Dict{DataType,Int32}(
    Marker => 0, Drift => 1, Quadrupole => 2, Sextupole => 3, Octupole => 4, ThinMultipole => 5,
    SBend => 6, ExactSBend => 7, RFCavity => 8, Solenoid => 9, Corrector => 10, Translation => 11,
    YRotation => 12, CrabCavity => 13, AccelCavity => 14, LongitudinalRFMap => 15, LorentzBoost => 16,
    InvLorentzBoost => 17, SpaceCharge => 18, DriftSC => 19, QuadrupoleSC => 20, SextupoleSC => 21,
    OctupoleSC => 22, SBendSC => 23, StrongThinGaussianBeam => 24, LBend => 25, Wiggler => 26,
    StrongGaussianBeam => 27, LongitudinalRLCWake => 28, LongitudinalWake => 29)

check(st, what) = st == 0 || error("$what: " * unsafe_string(ccall((:tp_strerror, LIB), Cstring, (Cint,), st)) *
                                   " (" * unsafe_string(ccall((:tp_last_error_string, LIB), Cstring, ())) * ")")

field(e, s, default) = hasproperty(e, s) ? Float64(getproperty(e, s)) : default
vec4(e, s) = hasproperty(e, s) ? NTuple{4,Float64}(getproperty(e, s)) : (0.0, 0.0, 0.0, 0.0)

_rf_k(rf::RFCavity) = 2pi * rf.freq / 2.99792458e8
_rf_k(rf) = hasproperty(rf, :k) ? Float64(rf.k) : 0.0
_rf_h(rf::CrabCavity) = 1.0
_rf_h(rf) = hasproperty(rf, :h) ? Float64(rf.h) : 1.0

"""The array fields of an element, appended to `aux` (include/trackpad_b200.h
lists the layout per kind); returns (offset, length) for iparam."""
function pack_arrays!(aux::Vector{Float64}, e)
    off = length(aux)
    if e isa StrongGaussianBeam
        n = max(e.nzslice, 0)
        append!(aux, [i <= length(e.zslice_npar) ? e.zslice_npar[i] : 1.0 / n for i in 1:n])
        append!(aux, [i <= length(e.xoffsets) ? e.xoffsets[i] : 0.0 for i in 1:n])
        append!(aux, [i <= length(e.yoffsets) ? e.yoffsets[i] : 0.0 for i in 1:n])
    elseif e isa LongitudinalWake
        append!(aux, Float64.(e.times)); append!(aux, Float64.(e.wakefields))
    elseif e isa Wiggler
        append!(aux, Float64[e.NHharm, e.NVharm, e.rad])
        append!(aux, Float64.(e.By[1:6e.NHharm])); append!(aux, Float64.(e.Bx[1:6e.NVharm]))
    end
    (Int32(off), Int32(length(aux) - off))
end

"""Pack one TrackPad element into the C record (fields by reference name)."""
function pack(e::AbstractElement, mis_index::Int32, aux::Vector{Float64} = Float64[])
    T = typeof(e).name.wrapper
    kind = get(TP_KIND, T, Int32(-1))
    kind < 0 && throw(ArgumentError("element $(T) has no device implementation"))
    k = e isa Quadrupole ? e.k1 : e isa Sextupole ? e.k2 : e isa Octupole ? e.k3 : 0.0
    p = zeros(8); ip = (Int32(0), Int32(0))
    gap = field(e, :gap, 0.0)
    if e isa Solenoid; p[1] = e.ks
    elseif e isa Corrector; p[1] = e.xkick; p[2] = e.ykick
    elseif e isa Translation; p[1:3] .= (e.dx, e.dy, e.ds)
    elseif e isa CrabCavity; p[1:4] .= (e.k, e.phi, e.errors[1], e.errors[2])
    elseif e isa AccelCavity; p[1:2] .= (e.k, e.phis)
    elseif e isa LongitudinalRFMap; p[1:3] .= (e.alphac, _rf_k(e.rf), _rf_h(e.rf))
    elseif e isa LorentzBoost; p[1:4] .= (e.angle, e.cosang, 0.0, e.tanang); ip = (Int32(e.mode), Int32(0))
    elseif e isa InvLorentzBoost; p[1:4] .= (e.angle, e.cosang, e.sinang, 0.0); ip = (Int32(e.mode), Int32(0))
    elseif e isa Union{QuadrupoleSC,SextupoleSC,OctupoleSC}; p[1:4] .= (e.k0, e.k1, e.k2, e.k3)
    elseif e isa StrongThinGaussianBeam; p[1:5] .= (e.amplitude, e.rmssizex, e.rmssizey, e.xoffset, e.yoffset)
    elseif e isa LBend; p[1:2] .= (e.K, e.by_error); gap = e.full_gap
    elseif e isa LongitudinalRLCWake; p[1:4] .= (e.freq, e.Rshunt, e.Q0, e.scale)
    elseif e isa StrongGaussianBeam; p[1:4] .= (e.charge, e.total_energy, e.beamsize[1], e.beamsize[2])
        ip = pack_arrays!(aux, e)
    elseif e isa LongitudinalWake; p[1:2] .= (e.fliphalf, e.scale); ip = pack_arrays!(aux, e)
    elseif e isa Wiggler; p[1:3] .= (e.lw, e.Bmax, e.energy); ip = pack_arrays!(aux, e)
    end
    TpElem(kind, Int32(hasproperty(e, :max_order) ? e.max_order : 0),
           Int32(hasproperty(e, :num_int_steps) ? e.num_int_steps : (e isa Wiggler ? e.Nsteps : 0)),
           Int32(hasproperty(e, :fringe_bend_entrance) ? e.fringe_bend_entrance : 0),
           Int32(hasproperty(e, :fringe_bend_exit) ? e.fringe_bend_exit : 0), mis_index, ip,
           field(e, :L, 0.0), Float64(k), field(e, :angle, 0.0), field(e, :e1, 0.0), field(e, :e2, 0.0),
           field(e, :fint1, 0.0), field(e, :fint2, 0.0), gap, field(e, :gk, 0.0),
           vec4(e, :polynom_a), vec4(e, :polynom_b),
           hasproperty(e, :kick_angle) ? NTuple{2,Float64}(e.kick_angle) : (0.0, 0.0),
           field(e, :volt, 0.0), field(e, :freq, 0.0), field(e, :h, 0.0), field(e, :lag, 0.0),
           field(e, :philag, 0.0), field(e, :energy, 0.0), NTuple{8,Float64}(p))
end

misaligned(e) = hasproperty(e, :t1) && !(iszero(e.t1) && iszero(e.t2) && iszero(e.r1) && iszero(e.r2))

"""Compile a Lattice into a tp_lattice handle (freed by a finalizer)."""
mutable struct DeviceLattice
    handle::Ptr{Cvoid}
end

function DeviceLattice(lat::Lattice; strengths = nothing)
    elems = TpElem[]; mis = TpMisalign[]; aux = Float64[]
    for e in lat.elements
        b = e isa TimeVaryingElement ? e.base : e
        idx = Int32(-1)
        if misaligned(b)
            push!(mis, TpMisalign(Tuple(b.t1), Tuple(b.t2), Tuple(vec(b.r1)), Tuple(vec(b.r2))))
            idx = Int32(length(mis) - 1)
        end
        push!(elems, pack(b, idx, aux))
    end
    if strengths !== nothing  # (element indices, values): the main strength k of those records
        for (i, k) in zip(strengths...)
            r = elems[i]
            elems[i] = TpElem(ntuple(j -> fieldname(TpElem, j) === :k ? Float64(k) : getfield(r, j),
                                     fieldcount(TpElem))...)
        end
    end
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve elems mis aux begin
        check(ccall((:tp_lattice_create_ex, LIB), Cint,
                    (Ptr{TpElem}, Int64, Ptr{TpMisalign}, Int64, Ptr{Float64}, Int64, Ref{Ptr{Cvoid}}),
                    elems, length(elems), isempty(mis) ? C_NULL : mis, length(mis),
                    isempty(aux) ? C_NULL : aux, length(aux), h), "tp_lattice_create_ex")
    end
    d = DeviceLattice(h[])
    finalizer(x -> ccall((:tp_lattice_destroy, LIB), Cint, (Ptr{Cvoid},), x.handle), d)
    d
end

"""Evaluate the timed fields of every turn into the library's per-turn schedule
(materialize of src/time_dependence.jl, once per element per turn)."""
function set_schedule!(d::DeviceLattice, lat::Lattice, time, dt_turn, turn0, nturns)
    names = Dict(:L => 0, :k1 => 1, :k2 => 1, :k3 => 1, :angle => 2, :e1 => 3, :e2 => 4, :volt => 5,
                 :freq => 6, :lag => 7, :philag => 8, :energy => 9, :num_int_steps => 10)
    fields = Int32[]; cols = Tuple{Int,Symbol}[]
    for (i, e) in enumerate(lat.elements)
        e isa TimeVaryingElement || continue
        for s in keys(e.updates)
            push!(fields, Int32(i - 1), Int32(names[s])); push!(cols, (i, s))
        end
    end
    isempty(cols) && return
    vals = zeros(Float64, length(cols), nturns)
    for t in 1:nturns
        ctx = TimeContext(Float64(time + (t - 1) * dt_turn); turn = turn0 + t - 1)
        for (j, (i, s)) in enumerate(cols)
            vals[j, t] = Float64(getproperty(materialize(lat.elements[i], ctx), s))
        end
    end
    check(ccall((:tp_lattice_set_schedule, LIB), Cint, (Ptr{Cvoid}, Ptr{Int32}, Int32, Int32, Int32, Ptr{Float64}),
                d.handle, fields, length(cols), turn0, nturns, vals), "tp_lattice_set_schedule")
end

const CTX = Ref{Ptr{Cvoid}}(C_NULL)
function context()
    if CTX[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:tp_ctx_create, LIB), Cint, (Cint, Ref{Ptr{Cvoid}}), CUDA.device().handle, h), "tp_ctx_create")
        CTX[] = h[]
    end
    CTX[]
end

opts(device::Bool; aperture = 0.0) =
    TpOpts(Int32(sizeof(TpOpts)), 1, device ? 1 : 0, 0, 0, 0, 0, 0, aperture, aperture,
           device ? Ptr{Cvoid}(CUDA.stream().handle) : C_NULL, 0, 0)

"""ringpass! on the GPU for device arrays: coords is N x 6 (column-major, as on the CPU)."""
function TrackPad.ringpass!(coords::CuMatrix{Float64}, lat::Lattice, beam::Beam{Float64},
                            lost_flags::CuVector{Int}, nturns::Int; time::Real = 0.0, dt_turn::Real = 0.0,
                            turn::Integer = 0, aperture::Real = 0.0)
    size(coords, 2) == 6 || throw(ArgumentError("coords must be N x 6"))
    d = DeviceLattice(lat)
    set_schedule!(d, lat, time, dt_turn, turn, max(nturns, 1))
    o = Ref(opts(true; aperture = Float64(aperture)))
    check(ccall((:tp_ringpass, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, CuPtr{Float64}, Int64, CuPtr{Int64}, Ptr{Int32}, Ptr{Int32}, Float64, Int32,
                 Float64, Float64, Int32, Ref{TpOpts}),
                context(), d.handle, coords, size(coords, 1), lost_flags, C_NULL, C_NULL, beti(beam), nturns,
                time, dt_turn, turn, o), "tp_ringpass")
    nothing
end

TrackPad.linepass!(coords::CuMatrix{Float64}, lat::Lattice, beam::Beam{Float64}, lost_flags::CuVector{Int};
                   time::Real = 0.0, turn::Integer = 0, aperture::Real = 0.0) =
    TrackPad.ringpass!(coords, lat, beam, lost_flags, 1; time = time, turn = turn, aperture = aperture)

"""Backend tag: B200() runs host arrays through the device (copies in and out)."""
struct B200 end

function TrackPad.ringpass!(::B200, coords::Matrix{Float64}, lat::Lattice, beam::Beam{Float64},
                            lost_flags::Vector{Int}, nturns::Int; time::Real = 0.0, dt_turn::Real = 0.0,
                            turn::Integer = 0, aperture::Real = 0.0)
    d = DeviceLattice(lat)
    set_schedule!(d, lat, time, dt_turn, turn, max(nturns, 1))
    o = Ref(opts(false; aperture = Float64(aperture)))
    GC.@preserve coords lost_flags begin
        check(ccall((:tp_ringpass, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Int64}, Ptr{Int32}, Ptr{Int32}, Float64, Int32,
                     Float64, Float64, Int32, Ref{TpOpts}),
                    context(), d.handle, coords, size(coords, 1), lost_flags, C_NULL, C_NULL, beti(beam), nturns,
                    time, dt_turn, turn, o), "tp_ringpass")
    end
    nothing
end

# --- Derivatives ---------------------------------------------------------------
"""
    loss_and_gradient(coords0, lat, beam, nturns, params; sigma, lost_weight = 1e3, ks = nothing, ...)

Loss of the tracked beam, mean over survivors of (x^2 + y^2)/sigma^2 plus
lost_weight x lost fraction, and its gradient with respect to the strength
(k1, k2, k3) of the Quadrupole/Sextupole/Octupole elements `params` (1-based
indices into `lat.elements`), from the B200 adjoint (tp_ringpass_adjoint).
`ks`, if given, replaces those strengths.  coords0 is read only.
"""
function loss_and_gradient(coords0::Matrix{Float64}, lat::Lattice, beam::Beam{Float64}, nturns::Int,
                           params::AbstractVector{<:Integer}; sigma::Real, lost_weight::Real = 1e3, ks = nothing,
                           aperture::Real = 0.0, time::Real = 0.0, dt_turn::Real = 0.0, turn::Integer = 0,
                           checkpoint_every::Integer = 0)
    size(coords0, 2) == 6 || throw(ArgumentError("coords0 must be N x 6"))
    d = DeviceLattice(lat; strengths = ks === nothing ? nothing : (params, ks))
    set_schedule!(d, lat, time, dt_turn, turn, max(nturns, 1))
    p0 = Int32[i - 1 for i in params]
    loss = Ref(0.0); grad = zeros(length(params))
    spec = Ref(TpLossSpec(0, 0, Float64(sigma), Float64(lost_weight)))
    o = Ref(opts(false; aperture = Float64(aperture)))
    GC.@preserve coords0 p0 grad begin
        check(ccall((:tp_ringpass_adjoint, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Int64}, Float64, Int32, Float64, Float64,
                     Int32, Ptr{Int32}, Int32, Ref{TpLossSpec}, Int32, Ref{Float64}, Ptr{Float64}, Ptr{Float64},
                     Ptr{Int64}, Ref{TpOpts}),
                    context(), d.handle, coords0, size(coords0, 1), C_NULL, beti(beam), nturns, time, dt_turn, turn,
                    p0, length(p0), spec, checkpoint_every, loss, grad, C_NULL, C_NULL, o), "tp_ringpass_adjoint")
    end
    loss[], grad
end

"""beam_loss(ks, coords0, lat, beam, nturns, params; sigma, ...): the loss alone,
differentiable in `ks` (ChainRulesCore rrule and Enzyme reverse rule in
TrackPadB200ADExt)."""
beam_loss(ks, coords0, lat, beam, nturns, params; kw...) =
    loss_and_gradient(coords0, lat, beam, nturns, params; ks = ks, kw...)[1]
# Positional form (sigma, lost_weight) for the Enzyme rule, whose arguments are annotated one by one.
beam_loss(ks, coords0, lat, beam, nturns, params, sigma::Real, lost_weight::Real) =
    loss_and_gradient(coords0, lat, beam, nturns, params; ks = ks, sigma = sigma, lost_weight = lost_weight)[1]

"""
    tangent_maps(lat, beam, orbits; nturns = 1) -> (M, err)

Exact tangent maps of `nturns` passes about each row of `orbits` (n x 6) and
their symplecticity error ||M'JM - J||, J = diag(J2, J2, -J2): the device
counterpart of one_turn_map (src/optics.jl:110-121, finite differences there).
"""
function tangent_maps(lat::Lattice, beam::Beam{Float64}, orbits::Matrix{Float64}; nturns::Int = 1, turn::Integer = 0)
    d = DeviceLattice(lat)
    set_schedule!(d, lat, 0.0, 0.0, turn, max(nturns, 1))
    n = size(orbits, 1)
    jac = zeros(36, n); err = zeros(n)
    o = Ref(opts(false))
    GC.@preserve orbits jac err begin
        check(ccall((:tp_one_turn_jacobian, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Int64, Float64, Int32, Int32, Ptr{Float64}, Ptr{Float64},
                     Ref{TpOpts}),
                    context(), d.handle, orbits, n, beti(beam), nturns, turn, jac, err, o), "tp_one_turn_jacobian")
    end
    [reshape(jac[:, i], 6, 6) for i in 1:n], err
end

"""
    taylor_maps(lat, beam, r0s; order = 1, nturns = 1, turn = 0) -> (coef, exps)

Truncated power series maps of `nturns` passes about each row of `r0s`
(`n x 6`): the device counterpart of `polyseries_one_turn_map`
(ext/TrackPadPolySeriesExt.jl:701-705) for many reference orbits at once.
`coef[k, c, i]` is the coefficient of monomial k (exponents `exps[:, k]`) in
component c of map i; a PolySeries CTPS is filled from it by exponents.
"""
function taylor_maps(lat::Lattice, beam::Beam{Float64}, r0s::Matrix{Float64}; order::Int = 1, nturns::Int = 1,
                     turn::Integer = 0)
    d = DeviceLattice(lat)
    set_schedule!(d, lat, 0.0, 0.0, turn, max(nturns, 1))
    m = Ref{Int64}(0)
    check(ccall((:tp_tpsa_coefficients, LIB), Cint, (Int32, Ref{Int64}), order, m), "tp_tpsa_coefficients")
    M = Int(m[])
    exps = zeros(Int32, 6, M)
    check(ccall((:tp_tpsa_monomials, LIB), Cint, (Int32, Ptr{Int32}), order, exps), "tp_tpsa_monomials")
    n = size(r0s, 1)
    coef = zeros(M, 6, n)                       # the C layout nmaps x 6 x M, column-major here
    for i in 1:n, c in 1:6
        coef[1, c, i] = r0s[i, c]
        coef[1 + c, c, i] = 1.0                 # CTPS(r0[c], c)
    end
    GC.@preserve coef begin
        check(ccall((:tp_tpsa_ringpass, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Int64, Int32, Float64, Int32, Int32),
                    context(), d.handle, coef, n, order, beti(beam), nturns, turn), "tp_tpsa_ringpass")
    end
    coef, exps
end

end # module
