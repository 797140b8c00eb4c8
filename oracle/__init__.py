"""CPU oracle for the 3-prime NTT multiplication path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs may
import this package, and only as the checker or as the timed CPU reference.  The product
package fast_mul_ntt_b200 never imports it.
"""
