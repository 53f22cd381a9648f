"""CPU oracle for the AD-TLERT 2.5D/3D forward-and-sensitivity path.

TEST INFRASTRUCTURE ONLY. Nothing in the product package may import, link or execute this
package: it is the checker that parity tests, the smoke check and the benchmark's CPU
baseline compare the CUDA path against. It restates the reference algorithm in NumPy/SciPy
(every function cites the reference ``file:line`` it follows) and is pinned by golden vectors
produced by the reference itself (``tests/golden/make_golden.py``).
"""
