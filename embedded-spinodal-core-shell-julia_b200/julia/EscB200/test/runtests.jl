# The identities of checks.jl:28-29 through the GPU loop; with CORE_SHELL_JL set
# to the path of core_shell.jl (FFTW installed), also the reference loop itself
# on the same inputs, with its own initial_fields (MersenneTwister noise).
const REF = get(ENV, "CORE_SHELL_JL", "")
isempty(REF) || include(REF)

using Test
using EscB200

# disc particle of core_shell.jl:29-30 and a mean-free noisy interior, from a
# small linear congruential generator (the reference's MersenneTwister stream
# is only used when the reference itself is loaded)
function disc_fields(n; radius=16.0, width=4.0, seed=1)
    phi = [0.5 * (1 - tanh((hypot(i - 1 - n ÷ 2, j - 1 - n ÷ 2) - radius) / width)) for i in 1:n, j in 1:n]
    state = UInt64(seed)
    noise = zeros(n, n)
    for k in eachindex(noise)
        state = state * 0x5851f42d4c957f2d + 0x14057b7ef767814f
        noise[k] = 0.01 * (2 * ((state >> 11) / 2.0^53) - 1)
    end
    inside = phi .>= 0.5
    noise .-= sum(noise[inside]) / count(inside)
    c = fill(0.5, n, n)
    c[inside] .+= noise[inside]
    return c, phi
end

@testset "EscB200" begin
    @test supported_size(64)
    c0, phi = isempty(REF) ? disc_fields(64) : initial_fields(64; radius=16.0)
    mean0 = sum(c0) / length(c0)
    c64, h64 = run_simulation_gpu(c0, phi; dt=0.01, steps=300, precision=ESC_FP64)
    @test size(h64) == (301, 6)
    @test h64[:, 1] ≈ 0.01 .* (0:300)
    @test maximum(abs.(h64[:, 2] .- mean0)) < 1e-12            # mass (checks.jl:28)
    @test maximum(diff(h64[:, 3])) < 1e-8                       # energy non-increasing (checks.jl:29)
    # mixed mode: FP64 state (mass kept to rounding), FP32 flux transforms
    c32, h32 = run_simulation_gpu(c0, phi; dt=0.01, steps=300, precision=ESC_MIXED)
    @test maximum(abs.(h32[:, 2] .- mean0)) < 1e-12
    @test maximum(abs.(h32[:, 3] .- h64[:, 3]) ./ abs.(h64[:, 3])) < 1e-5
    @test maximum(abs.(c32 .- c64)) < 1e-4 * maximum(abs.(c64))
    if !isempty(REF)
        c, h = run_simulation_gpu(c0, phi; dt=0.01, steps=300)
        cr, hr = run_simulation(c0, phi; dt=0.01, steps=300)
        @test maximum(abs.(c .- cr)) <= 1e-12 * maximum(abs.(cr))
        for j in 1:6
            @test maximum(abs.(h[:, j] .- hr[:, j])) <= 1e-12 * max(maximum(abs.(hr[:, j])), 1e-300)
        end
    end
    bad = copy(c0)
    bad[3, 4] = NaN
    @test_throws ErrorException run_simulation_gpu(bad, phi; steps=5)
    cs, hs, flags = run_batch_gpu([c0, bad], [phi, phi]; steps=20, precision=ESC_FP64)
    @test flags == [-1, 0]
    @test isequal(cs[2], bad)                                 # a failed particle's field is left unchanged
    c1, h1 = run_simulation_gpu(c0, phi; steps=20)
    @test maximum(abs.(cs[1] .- c1)) <= 1e-12 * maximum(abs.(c1))
    L, dc0, dtheta = esc_adjoint_call(c0, phi, c1; steps=40, precision=ESC_FP64)
    @test isfinite(L) && size(dc0) == (64, 64) && length(dtheta) == 4
end
