"""CPU oracle for the cupbr rendering hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may import it.
"""
