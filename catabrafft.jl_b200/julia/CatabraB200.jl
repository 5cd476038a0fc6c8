# CatabraB200.jl -- Julia binding of libcatabra_b200.so (include/catabra_b200.h).
#
# Drop-in for the reference's public FFT API (src/CatabraFFT.jl:39-196):
# fft / ifft / bfft / fft! / plan_fft / mul! / * / empty_cache, with the same
# FLAG values (src/spells.jl:4-8).  Host Vector{Complex{T}} buffers go through
# cfft_execute_host (copy in, transform on the GPU, copy out).  Julia is not
# installed on the machines of this build, so this file is untested here; the
# same C entry points are exercised from Python (tests/).
module CatabraB200

import LinearAlgebra: mul!
import Base: *

const LIB = get(ENV, "CATABRA_B200_LIB", joinpath(@__DIR__, "..", "libcatabra_b200.so"))

const FLAG = Int8
const NO_FLAG = FLAG(0)
const MEASURE = FLAG(1)
const ENCHANT = FLAG(2)

const CFFT_FORWARD, CFFT_INVERSE, CFFT_BACKWARD = Cint(0), Cint(1), Cint(2)

dtype_code(::Type{Float64}) = Cint(0)
dtype_code(::Type{Float32}) = Cint(1)

function check(rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:cfft_last_error, LIB), Cstring, ()))
    error("catabra_b200 error $rc: $msg")
end

mutable struct Spell{T<:AbstractFloat}
    n::Int
    datatype::Type{T}
    flag::FLAG
    handle::Ptr{Cvoid}
    function Spell(n::Int, ::Type{T}, flag::FLAG) where {T<:Union{Float32,Float64}}
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:cfft_plan_create, LIB), Cint,
                    (Ref{Ptr{Cvoid}}, Int64, Int64, Cint, Cint),
                    h, n, 1, dtype_code(T), Cint(flag)))
        p = new{T}(n, T, flag, h[])
        finalizer(p) do q
            q.handle != C_NULL && ccall((:cfft_plan_destroy, LIB), Cint, (Ptr{Cvoid},), q.handle)
            q.handle = C_NULL
        end
        return p
    end
end

# plan cache, the counterpart of F_cache (src/kernel.jl:12-51)
const PLANS = Dict{Tuple{Int,DataType,FLAG},Spell}()
getplan(n::Int, ::Type{T}, flag::FLAG) where {T} = get!(() -> Spell(n, T, flag), PLANS, (n, T, flag))

function run!(y::Vector{Complex{T}}, p::Spell{T}, x::Vector{Complex{T}}, dir::Cint) where {T}
    length(x) == p.n == length(y) || throw(DimensionMismatch("plan is for n=$(p.n)"))
    check(ccall((:cfft_execute_host, LIB), Cint, (Ptr{Cvoid}, Ptr{Complex{T}}, Ptr{Complex{T}}, Cint),
                p.handle, x, y, dir))
    return y
end

fft(x::Vector{Complex{T}}) where {T<:Union{Float32,Float64}} =
    run!(similar(x), getplan(length(x), T, NO_FLAG), x, CFFT_FORWARD)
ifft(x::Vector{Complex{T}}) where {T<:Union{Float32,Float64}} =
    run!(similar(x), getplan(length(x), T, NO_FLAG), x, CFFT_INVERSE)
bfft(x::Vector{Complex{T}}) where {T<:Union{Float32,Float64}} =
    run!(similar(x), getplan(length(x), T, NO_FLAG), x, CFFT_BACKWARD)
fft!(x::Vector{Complex{T}}) where {T<:Union{Float32,Float64}} =
    run!(x, getplan(length(x), T, NO_FLAG), x, CFFT_FORWARD)

plan_fft(x::Vector{Complex{T}}, flags::FLAG=NO_FLAG) where {T} = getplan(length(x), T, flags)
mul!(y::Vector{Complex{T}}, p::Spell{T}, x::Vector{Complex{T}}) where {T} = run!(y, p, x, CFFT_FORWARD)
*(p::Spell{T}, x::Vector{Complex{T}}) where {T} = run!(similar(x), p, x, CFFT_FORWARD)

function empty_cache()
    for p in values(PLANS)
        finalize(p)
    end
    empty!(PLANS)
    check(ccall((:cfft_empty_cache, LIB), Cint, ()))
end

end # module
