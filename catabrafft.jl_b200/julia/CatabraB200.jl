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
dtype_code(::Type{Float16}) = Cint(2)     # ComplexF16 data, FP32 arithmetic

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
    function Spell(n::Int, ::Type{T}, flag::FLAG) where {T<:Union{Float16,Float32,Float64}}
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

const Fl = Union{Float16,Float32,Float64}
fft(x::Vector{Complex{T}}) where {T<:Fl} = run!(similar(x), getplan(length(x), T, NO_FLAG), x, CFFT_FORWARD)
ifft(x::Vector{Complex{T}}) where {T<:Fl} = run!(similar(x), getplan(length(x), T, NO_FLAG), x, CFFT_INVERSE)
bfft(x::Vector{Complex{T}}) where {T<:Fl} = run!(similar(x), getplan(length(x), T, NO_FLAG), x, CFFT_BACKWARD)
fft!(x::Vector{Complex{T}}) where {T<:Fl} = run!(x, getplan(length(x), T, NO_FLAG), x, CFFT_FORWARD)

plan_fft(x::Vector{Complex{T}}, flags::FLAG=NO_FLAG) where {T} = getplan(length(x), T, flags)
mul!(y::Vector{Complex{T}}, p::Spell{T}, x::Vector{Complex{T}}) where {T} = run!(y, p, x, CFFT_FORWARD)
*(p::Spell{T}, x::Vector{Complex{T}}) where {T} = run!(similar(x), p, x, CFFT_FORWARD)

# real input: rfft / irfft / brfft (AbstractFFTs semantics; plan_rfft and
# plan_brfft are stubs in the reference, src/CatabraFFT.jl:199-209)
mutable struct RSpell{T<:AbstractFloat}
    n::Int
    handle::Ptr{Cvoid}
    function RSpell(n::Int, ::Type{T}, flag::FLAG) where {T<:Union{Float32,Float64}}
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:cfft_rfft_plan_create, LIB), Cint, (Ref{Ptr{Cvoid}}, Int64, Int64, Cint, Cint),
                    h, n, 1, dtype_code(T), Cint(flag)))
        p = new{T}(n, h[])
        finalizer(p) do q
            q.handle != C_NULL && ccall((:cfft_rfft_plan_destroy, LIB), Cint, (Ptr{Cvoid},), q.handle)
            q.handle = C_NULL
        end
        return p
    end
end
const RPLANS = Dict{Tuple{Int,DataType,FLAG},RSpell}()
getrplan(n::Int, ::Type{T}, flag::FLAG) where {T} = get!(() -> RSpell(n, T, flag), RPLANS, (n, T, flag))

function rfft(x::Vector{T}) where {T<:Union{Float32,Float64}}
    p = getrplan(length(x), T, NO_FLAG)
    y = Vector{Complex{T}}(undef, length(x) ÷ 2 + 1)
    check(ccall((:cfft_rfft_execute_host, LIB), Cint, (Ptr{Cvoid}, Ptr{T}, Ptr{Complex{T}}, Cint),
                p.handle, x, y, CFFT_FORWARD))
    return y
end
function _c2r(X::Vector{Complex{T}}, d::Int, dir::Cint) where {T<:Union{Float32,Float64}}
    length(X) == d ÷ 2 + 1 || throw(DimensionMismatch("expected $(d ÷ 2 + 1) values for d=$d"))
    p = getrplan(d, T, NO_FLAG)
    y = Vector{T}(undef, d)
    check(ccall((:cfft_rfft_execute_host, LIB), Cint, (Ptr{Cvoid}, Ptr{Complex{T}}, Ptr{T}, Cint),
                p.handle, X, y, dir))
    return y
end
irfft(X::Vector{Complex{T}}, d::Integer) where {T} = _c2r(X, Int(d), CFFT_INVERSE)
brfft(X::Vector{Complex{T}}, d::Integer) where {T} = _c2r(X, Int(d), CFFT_BACKWARD)

# wisdom: MEASURE / ENCHANT choices across sessions (the serialisable Spell
# the reference sketched in src/spells.jl:180-375)
export_wisdom(path::AbstractString) = check(ccall((:cfft_wisdom_export, LIB), Cint, (Cstring,), path))
import_wisdom(path::AbstractString) = check(ccall((:cfft_wisdom_import, LIB), Cint, (Cstring,), path))
forget_wisdom() = check(ccall((:cfft_wisdom_forget, LIB), Cint, ()))

# the device fault word: 0 unless a kernel's bounded wait gave up (bit 0: a
# tensor copy, bit 1: a work-queue or dataflow dependency); that launch's
# results are then incomplete
device_faults(clear::Bool = false) = ccall((:cfft_device_faults, LIB), Cint, (Cint,), clear ? 1 : 0)

# batched form: many transforms of mixed lengths packed back to back in one
# device buffer (pointers from CUDA.jl, e.g. `pointer(x)` of a CuVector),
# one graph launch of the work-queue kernel per execution
const BATCH_GROUPED = Cint(32)
mutable struct Batch
    lengths::Vector{Int64}
    handle::Ptr{Cvoid}
    function Batch(lengths::Vector{Int64}, ::Type{T}; grouped::Bool = false) where {T<:Union{Float32,Float64}}
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:cfft_batch_create, LIB), Cint, (Ref{Ptr{Cvoid}}, Int64, Ptr{Int64}, Cint, Cint),
                    h, length(lengths), lengths, dtype_code(T), grouped ? BATCH_GROUPED : Cint(0)))
        b = new(copy(lengths), h[])
        finalizer(b) do b
            b.handle == C_NULL || ccall((:cfft_batch_destroy, LIB), Cint, (Ptr{Cvoid},), b.handle)
            b.handle = C_NULL
        end
        return b
    end
end
execute!(b::Batch, d_out::Ptr{Cvoid}, d_in::Ptr{Cvoid}, dir::Cint = CFFT_FORWARD, stream::Ptr{Cvoid} = C_NULL) =
    check(ccall((:cfft_batch_execute, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Cvoid}),
                b.handle, d_in, d_out, dir, stream))

function empty_cache()
    for p in values(PLANS)
        finalize(p)
    end
    empty!(PLANS)
    for p in values(RPLANS)
        finalize(p)
    end
    empty!(RPLANS)
    check(ccall((:cfft_empty_cache, LIB), Cint, ()))
end

end # module
