# Project-written probe compiled against the reference's .pxd declarations
# (TEST INFRASTRUCTURE): exposes the reference's cdef special functions and
# random-number wrappers (specFun.pyx, randomGen.pyx) to Python so that
# golden vectors can be generated from them.
cimport specFun
cimport randomGen

def betaincinv(double a, double b, double p):
    return specFun.betaincinv(a, b, p)

def gammaincinv(double a, double p):
    return specFun.gammaincinv(a, p)

def gammainc(double a, double x):
    return specFun.gammainc(a, x)

def betainc(double a, double b, double x):
    return specFun.betainc(a, b, x)

def binom(unsigned int k, double p, unsigned int n):
    return specFun.binom(k, p, n)

def rand():
    return randomGen.rand()

def randn():
    return randomGen.randn()

def randi(unsigned long n):
    return randomGen.randi(n)
