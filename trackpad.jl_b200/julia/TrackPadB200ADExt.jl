"""
    TrackPadB200ADExt

Differentiation rules for `TrackPadB200Ext.beam_loss`, backed by the B200
adjoint (tp_ringpass_adjoint): a ChainRulesCore `rrule` (keyword form) and an
Enzyme reverse rule (positional form beam_loss(ks, coords0, lat, beam, nturns,
params, sigma, lost_weight), Duplicated ks, everything else Const).  Both return d loss / d ks from one forward + one reverse launch, with
the survivor set of the forward pass held fixed.

Registration in TrackPad's Project.toml:
    [weakdeps]    ChainRulesCore = "d360d2e6-b24c-11e9-a2a3-2a2ae2dbcce4"
                  EnzymeCore = "f151be2c-9106-41f4-ab19-57ee4f262869"
    [extensions]  TrackPadB200ADExt = ["CUDA", "ChainRulesCore", "EnzymeCore"]
"""
module TrackPadB200ADExt

using TrackPad
using ChainRulesCore
using EnzymeCore
using EnzymeCore: EnzymeRules

const B = Base.get_extension(TrackPad, :TrackPadB200Ext)

function ChainRulesCore.rrule(::typeof(B.beam_loss), ks::AbstractVector{<:Real}, coords0, lat, beam, nturns, params;
                              kw...)
    loss, grad = B.loss_and_gradient(coords0, lat, beam, nturns, params; ks = ks, kw...)
    beam_loss_pullback(dl) = (NoTangent(), unthunk(dl) .* grad, NoTangent(), NoTangent(), NoTangent(), NoTangent(),
                              NoTangent())
    return loss, beam_loss_pullback
end

function EnzymeRules.augmented_primal(config, ::EnzymeCore.Const{typeof(B.beam_loss)},
                                      ::Type{<:EnzymeCore.Active}, ks::EnzymeCore.Duplicated,
                                      coords0::EnzymeCore.Const, lat::EnzymeCore.Const, beam::EnzymeCore.Const,
                                      nturns::EnzymeCore.Const, params::EnzymeCore.Const, sigma::EnzymeCore.Const,
                                      lost_weight::EnzymeCore.Const)
    loss, grad = B.loss_and_gradient(coords0.val, lat.val, beam.val, nturns.val, params.val; ks = ks.val,
                                     sigma = sigma.val, lost_weight = lost_weight.val)
    primal = EnzymeRules.needs_primal(config) ? loss : nothing
    return EnzymeRules.AugmentedReturn(primal, nothing, grad)
end

function EnzymeRules.reverse(config, ::EnzymeCore.Const{typeof(B.beam_loss)}, dret::EnzymeCore.Active, grad,
                             ks::EnzymeCore.Duplicated, coords0, lat, beam, nturns, params, sigma, lost_weight)
    ks.dval .+= dret.val .* grad
    return (nothing, nothing, nothing, nothing, nothing, nothing, nothing, nothing)
end

end # module
