"""B200-native enumerative LTL learner (characteristic-set enumeration on sm_100a)."""
