"""Restatement of the device DE rule (forcesmith_b200/csrc/population.cu) in
Python integers and IEEE doubles, for bit-exact checks of one generation.

Random numbers: u(seed, gen, i, draw) = top 53 bits of
mix(seed ^ mix(gen·0x100000001B3 ^ mix(i·0x9E3779B1 + draw))) · 2⁻⁵³, with
mix the SplitMix64 finaliser; draws 0,1,… pick r1, r2, r3 (rejecting i and
repeats; after 64 draws for one parent, the first free index), draw 2³³ picks the forced coordinate, draw 2³² + j decides
crossover of coordinate j; the initial population uses gen = 2³² − 1 and
draw j.
"""
import numpy as np

M64 = (1 << 64) - 1


def mix64(z):
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def urand(seed, gen, i, draw):
    inner = mix64((i * 0x9E3779B1 + draw) & M64)
    z = mix64(seed ^ mix64(((gen * 0x100000001B3) & M64) ^ inner))
    return (z >> 11) * (1.0 / 9007199254740992.0)


def de_init_population(seed, lo, hi, x0, NP):
    D = len(lo)
    pop = np.zeros((NP, D))
    for i in range(NP):
        for j in range(D):
            if i == 0 and x0 is not None:
                pop[i, j] = min(max(float(x0[j]), float(lo[j])), float(hi[j]))
            else:
                pop[i, j] = float(lo[j]) + (float(hi[j]) - float(lo[j])) * urand(seed, 0xFFFFFFFF, i, j)
    return pop


def de_trials(seed, gen, pop, lo, hi, F, CR):
    NP, D = pop.shape
    out = np.zeros_like(pop)
    for i in range(NP):
        r = []
        draw = 0
        for _ in range(3):
            c = -1
            for _t in range(64):
                v = min(int(urand(seed, gen, i, draw) * NP), NP - 1)
                draw += 1
                if v != i and v not in r:
                    c = v
                    break
            if c < 0:
                c = next(v for v in range(NP) if v != i and v not in r)
            r.append(c)
        jr = min(int(urand(seed, gen, i, 1 << 33) * D), D - 1)
        for j in range(D):
            if j == jr or urand(seed, gen, i, (1 << 32) + j) < CR:
                v = float(pop[r[0], j]) + F * (float(pop[r[1], j]) - float(pop[r[2], j]))
                out[i, j] = min(max(v, float(lo[j])), float(hi[j]))
            else:
                out[i, j] = pop[i, j]
    return out
