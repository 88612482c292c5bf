"""CPU oracle for the bitstream executor -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and the CPU-baseline legs of
bench.py.  The product (bitstreamzoo_b200, libbsz) never imports it.
"""
