"""
Reverse-mode rule for `EscB200.calibration_loss`: the pullback scales the
gradients that the library's FP64 adjoint returns (`esc_adjoint`, one call for
the loss and both gradients).  Gradients with respect to the particle φ and to
the target field are not computed by the library and are marked as such.
"""
module EscB200ChainRulesCoreExt

using EscB200: EscB200, calibration_loss, loss_and_gradients
using ChainRulesCore: ChainRulesCore, NoTangent, @not_implemented, unthunk

function ChainRulesCore.rrule(::typeof(calibration_loss), c0, theta, phi, c_target; kw...)
    L, dc0, dtheta = loss_and_gradients(c0, theta, phi, c_target; kw...)
    function calibration_loss_pullback(dL)
        s = unthunk(dL)
        return (NoTangent(), s .* dc0, s .* dtheta,
                @not_implemented("libesc computes no gradient with respect to phi"),
                @not_implemented("libesc computes no gradient with respect to c_target"))
    end
    return L, calibration_loss_pullback
end

end # module
